/* placeholder, replaced by the Cornelius cube scan */
#include "vh_kernels.h"
namespace vh {
size_t freezeout_scratch_ints(int nx, int ny, int nz) { return 8; }
__global__ void fo_stub(int *hdr) { hdr[0] = 0; hdr[1] = 0; }
void launch_freezeout(const FoArgs &a, cudaStream_t s) { fo_stub<<<1, 1, 0, s>>>(a.counts + 6); }
}
