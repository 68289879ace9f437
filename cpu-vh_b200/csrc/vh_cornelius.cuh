/*
 * vh_cornelius.cuh -- the Cornelius 1.3 iso-surface construction for one
 * cube (2+1D hydro) or hypercube (3+1D hydro), as device code run by one
 * thread.  Algorithm of P. Huovinen and H. Petersen (arXiv:1206.3371), as the
 * reference uses it through freezeout/cornelius-c++-1.3/cornelius.cpp:
 * edges are cut linearly (with the 1e-9 nudges for corners exactly on the
 * threshold), cuts become lines per square face, lines chain into polygons per
 * cube face (with the ambiguity rules), polygons join into polyhedra per
 * hypercube; centroids are area/volume-weighted sums over triangles/tetrahedra
 * and normals are the outward-oriented sums of their normals.  Every sum runs
 * in the reference's order so the element geometry is identical bit for bit.
 *
 * Storage is fixed-size: lines are kept once (12 doubles each) and
 * polygons/polyhedra refer to them by index, through a WorkRef (a view of
 * one thread's Work).  Capacities are the reference's own array bounds
 * (cornelius.h: 2 lines per square, 8 polygons per cube, 10 polyhedra per
 * hypercube, 24 lines per polygon and 24 polygons per polyhedron); exceeding
 * one raises an error instead of overrunning.
 *
 * MODIFIED VERSION of the Cornelius subroutine: restated in 2026 as CUDA
 * device code (one thread per cube or hypercube, fixed-size per-thread
 * storage, status codes instead of exit()), with the same arithmetic.  The
 * original copyright and permission notice follows; this file is
 * distributed under the same terms.
 *
 * cornelius version 1.3: Copyright 2012, Pasi Huovinen
 *
 * This subroutine is aimed to be used as a part of the fluid dynamical
 * models of the heavy-ion physics community. Permission to use it for
 * any purpose except for any commercial purpose is granted, provided
 * that any publication cites the paper describing the algorithm:
 * P. Huovinen and H. Petersen, arXiv:1206.3371 [nucl-th].
 *
 * Permission to distribute this subroutine is granted, provided that no
 * fee is charged, and that this copyright and permission notice appear
 * in all the copies. Permission to modify this subroutine is granted
 * provided that the modified subroutine is made publicly available
 * latest when any results obtained using the modified subroutine are
 * published, the modified subroutine is distributed under terms similar
 * to this notice, and the modified code carries both the original
 * copyright notice and notices stating that you modified it, and a
 * relevant date/year.
 *
 * This program is distributed in the hope that it will be useful, but
 * WITHOUT ANY WARRANTY; without even the implied warranty of FITNESS FOR
 * A PARTICULAR PURPOSE.
 */
#ifndef VH_CORNELIUS_CUH
#define VH_CORNELIUS_CUH

namespace vh {
namespace cor {

constexpr int D = 4;
constexpr int kMaxLines = 96;     /* 8 cubes x 6 squares x 2 lines */
constexpr int kMaxPoly = 32;      /* polygons over the 8 cubes of a hypercube */
constexpr int kMaxPolyLines = 12; /* lines of one polygon: at most the lines of its cube */
constexpr int kMaxHedra = 10;     /* Hypercube MAX_POLY, cornelius.cpp:1703 */
constexpr int kMaxElements = 10;  /* Cornelius MAX_ELEMENTS, cornelius.cpp:2004 */

struct Poly {
    unsigned short line[kMaxPolyLines];   /* line indices (a block's shared pool may hold 512) */
    int nlines, const_i, x1, x2, x3;
    double cen[D];
    bool have_cen;
};

/* one thread's storage for a whole (hyper)cube */
struct Work {
    double p[kMaxLines][2][D];
    double out[kMaxLines][D];
    unsigned char flip[kMaxLines];
    Poly poly[kMaxPoly];
};

/* a view of line and polygon storage; nl and np count what was appended */
struct WorkRef {
    double (*p)[2][D];
    double (*out)[D];
    unsigned char *flip;
    Poly *poly;
    int nl, np, lcap, pcap;
    bool error;
};

__device__ __forceinline__ WorkRef work_ref(Work &w)
{
    return WorkRef{w.p, w.out, w.flip, w.poly, 0, 0, kMaxLines, kMaxPoly, false};
}

__device__ __forceinline__ const double *lstart(const WorkRef &w, int l) { return w.p[l][w.flip[l]]; }
__device__ __forceinline__ const double *lend(const WorkRef &w, int l) { return w.p[l][1 - w.flip[l]]; }

/* GeneralElement::check_normal_direction, cornelius.cpp:91-106 */
__device__ __forceinline__ void orient(double *n, const double *out)
{
    double dot = 0;
    for (int i = 0; i < D; i++) dot += out[i] * n[i];
    if (dot < 0)
        for (int i = 0; i < D; i++) n[i] = -n[i];
}

/* The number of edge cuts square_lines finds (0, 2 or 4; anything else is
 * its error), from the same comparisons, without computing the cuts: a
 * cube's line count before its lines are built. */
__device__ __forceinline__ int square_cut_count(const double P[2][2], double E0)
{
    int above = 0;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            if (P[i][j] >= E0) above++;
    if (above == 0 || above == 4) return 0;
    int nc = 0;
    if ((P[0][0] - E0) * (P[1][0] - E0) < 0) nc++;
    else if (P[0][0] == E0 && P[1][0] < E0) nc++;
    else if (P[1][0] == E0 && P[0][0] < E0) nc++;
    if ((P[0][0] - E0) * (P[0][1] - E0) < 0) nc++;
    else if (P[0][0] == E0 && P[0][1] < E0) nc++;
    else if (P[0][1] == E0 && P[0][0] < E0) nc++;
    if ((P[1][0] - E0) * (P[1][1] - E0) < 0) nc++;
    else if (P[1][0] == E0 && P[1][1] < E0) nc++;
    else if (P[1][1] == E0 && P[1][0] < E0) nc++;
    if ((P[0][1] - E0) * (P[1][1] - E0) < 0) nc++;
    else if (P[0][1] == E0 && P[1][1] < E0) nc++;
    else if (P[1][1] == E0 && P[0][1] < E0) nc++;
    return nc;
}

/* Square::construct_lines with ends_of_edge and find_outside
 * (cornelius.cpp:1134-1337); appends its lines to w. */
static __device__ void square_lines(WorkRef &w, const double P[2][2], int c0, int c1, double v0_, double v1_, double E0, const double *dx)
{
    int above = 0;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            if (P[i][j] >= E0) above++;
    if (above == 0 || above == 4) return;
    int x1 = -1, x2 = -1;
    for (int i = 0; i < D; i++)
        if (i != c0 && i != c1) { if (x1 < 0) x1 = i; else x2 = i; }
    const double d1 = dx[x1], d2 = dx[x2];
    double cuts[4][2], out[2][2];
    int nc = 0;
#define CUT(a, b) do { cuts[nc][0] = (a); cuts[nc][1] = (b); nc++; } while (0)
    if ((P[0][0] - E0) * (P[1][0] - E0) < 0) CUT((P[0][0] - E0) / (P[0][0] - P[1][0]) * d1, 0);
    else if (P[0][0] == E0 && P[1][0] < E0) CUT(1e-9 * d1, 0);
    else if (P[1][0] == E0 && P[0][0] < E0) CUT((1.0 - 1e-9) * d1, 0);
    if ((P[0][0] - E0) * (P[0][1] - E0) < 0) CUT(0, (P[0][0] - E0) / (P[0][0] - P[0][1]) * d2);
    else if (P[0][0] == E0 && P[0][1] < E0) CUT(0, 1e-9 * d2);
    else if (P[0][1] == E0 && P[0][0] < E0) CUT(0, (1.0 - 1e-9) * d2);
    if ((P[1][0] - E0) * (P[1][1] - E0) < 0) CUT(d1, (P[1][0] - E0) / (P[1][0] - P[1][1]) * d2);
    else if (P[1][0] == E0 && P[1][1] < E0) CUT(d1, 1e-9 * d2);
    else if (P[1][1] == E0 && P[1][0] < E0) CUT(d1, (1.0 - 1e-9) * d2);
    if ((P[0][1] - E0) * (P[1][1] - E0) < 0) CUT((P[0][1] - E0) / (P[0][1] - P[1][1]) * d1, d2);
    else if (P[0][1] == E0 && P[1][1] < E0) CUT(1e-9 * d1, d2);
    else if (P[1][1] == E0 && P[0][1] < E0) CUT((1.0 - 1e-9) * d1, d2);
#undef CUT
    if (nc != 0 && nc != 2 && nc != 4) { w.error = true; return; }
    if (nc == 0) return;
    bool ambiguous = false;
    if (nc == 4) {
        ambiguous = true;
        double Emid = 0;
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) Emid += 0.25 * P[i][j];
        if ((P[0][0] < E0 && Emid < E0) || (P[0][0] > E0 && Emid > E0))
            for (int i = 0; i < 2; i++) { double t = cuts[1][i]; cuts[1][i] = cuts[2][i]; cuts[2][i] = t; }
        if ((Emid - E0) < 0) {
            out[0][0] = out[1][0] = 0.5 * d1;
            out[0][1] = out[1][1] = 0.5 * d2;
        } else if ((P[0][0] - E0) < 0) {
            out[0][0] = 0; out[0][1] = 0; out[1][0] = d1; out[1][1] = d2;
        } else {
            out[0][0] = d1; out[0][1] = 0; out[1][0] = 0; out[1][1] = d2;
        }
    } else {
        out[0][0] = out[0][1] = out[1][0] = out[1][1] = 0;
        int nout = 0;
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++)
                if (P[i][j] < E0) { out[0][0] += i * d1; out[0][1] += j * d2; nout++; }
        if (nout > 0)
            for (int i = 0; i < 2; i++)
                for (int j = 0; j < 2; j++) out[i][j] = out[i][j] / (double)nout;
    }
    (void)ambiguous;
    for (int k = 0; k < nc / 2; k++) {
        if (w.nl >= w.lcap) { w.error = true; return; }
        int l = w.nl++;
        for (int e = 0; e < 2; e++) {
            w.p[l][e][x1] = cuts[2 * k + e][0];
            w.p[l][e][x2] = cuts[2 * k + e][1];
            w.p[l][e][c0] = v0_;
            w.p[l][e][c1] = v1_;
        }
        w.out[l][x1] = out[k][0];
        w.out[l][x2] = out[k][1];
        w.out[l][c0] = v0_;
        w.out[l][c1] = v1_;
        w.flip[l] = 0;
    }
}

__device__ __forceinline__ void poly_init(Poly &p, int c)
{
    p.const_i = c;
    p.x1 = p.x2 = p.x3 = -1;
    for (int i = 0; i < D; i++)
        if (i != c) { if (p.x1 < 0) p.x1 = i; else if (p.x2 < 0) p.x2 = i; else p.x3 = i; }
    p.nlines = 0;
    p.have_cen = false;
}

/* Polygon::add_line, cornelius.cpp:436-471 */
__device__ __forceinline__ bool poly_add_line(WorkRef &w, Poly &p, int l, bool donotcheck)
{
    if (donotcheck || p.nlines == 0) {
        if (p.nlines >= kMaxPolyLines) { w.error = true; return false; }
        p.line[p.nlines++] = (unsigned short)l;
        return true;
    }
    const double *p1 = lstart(w, l), *p2 = lend(w, l), *p3 = lend(w, p.line[p.nlines - 1]);
    double diff1 = 0, diff2 = 0;
    for (int j = 0; j < D; j++) { diff1 += fabs(p1[j] - p3[j]); diff2 += fabs(p2[j] - p3[j]); }
    if (diff1 < 1e-10 || diff2 < 1e-10) {
        if (diff2 < 1e-10) w.flip[l] ^= 1;
        if (p.nlines >= kMaxPolyLines) { w.error = true; return false; }
        p.line[p.nlines++] = (unsigned short)l;
        return true;
    }
    return false;
}

/* Polygon::calculate_centroid, cornelius.cpp:478-551 (pow(x, 2.0) is x*x:
 * the host libm returns the correctly rounded square) */
static __device__ const double *poly_centroid(const WorkRef &w, Poly &p)
{
    if (p.have_cen) return p.cen;
    double mean[D] = {0, 0, 0, 0};
    for (int i = 0; i < p.nlines; i++) {
        const double *p1 = lstart(w, p.line[i]), *p2 = lend(w, p.line[i]);
        for (int j = 0; j < D; j++) mean[j] += p1[j] + p2[j];
    }
    for (int j = 0; j < D; j++) mean[j] = mean[j] / (double)(2.0 * p.nlines);
    if (p.nlines == 3) {
        for (int i = 0; i < D; i++) p.cen[i] = mean[i];
        p.have_cen = true;
        return p.cen;
    }
    double up[D] = {0, 0, 0, 0}, down = 0;
    for (int i = 0; i < p.nlines; i++) {
        const double *p1 = lstart(w, p.line[i]), *p2 = lend(w, p.line[i]);
        double cm[D], a[D], b[D];
        for (int j = 0; j < D; j++) cm[j] = (p1[j] + p2[j] + mean[j]) / 3.0;
        for (int j = 0; j < D; j++) { a[j] = p1[j] - mean[j]; b[j] = p2[j] - mean[j]; }
        double s1 = a[p.x2] * b[p.x3] - a[p.x3] * b[p.x2];
        double s2 = a[p.x1] * b[p.x3] - a[p.x3] * b[p.x1];
        double s3 = a[p.x2] * b[p.x1] - a[p.x1] * b[p.x2];
        double A = 0.5 * sqrt(s1 * s1 + s2 * s2 + s3 * s3);
        for (int j = 0; j < D; j++) up[j] += cm[j] * A;
        down += A;
    }
    for (int i = 0; i < D; i++) p.cen[i] = up[i] / down;
    p.have_cen = true;
    return p.cen;
}

/* Polygon::calculate_normal, cornelius.cpp:559-617 */
static __device__ void poly_normal(const WorkRef &w, Poly &p, double *normal)
{
    const double *cen = poly_centroid(w, p);
    for (int i = 0; i < D; i++) normal[i] = 0;
    double acc[kMaxPolyLines][D];
    for (int i = 0; i < p.nlines; i++) {
        const double *p1 = lstart(w, p.line[i]), *p2 = lend(w, p.line[i]);
        double a[D], b[D], n[D], vout[D];
        for (int j = 0; j < D; j++) { a[j] = p1[j] - cen[j]; b[j] = p2[j] - cen[j]; n[j] = 0; }
        n[p.x1] = 0.5 * (a[p.x2] * b[p.x3] - a[p.x3] * b[p.x2]);
        n[p.x2] = -0.5 * (a[p.x1] * b[p.x3] - a[p.x3] * b[p.x1]);
        n[p.x3] = 0.5 * (a[p.x1] * b[p.x2] - a[p.x2] * b[p.x1]);
        n[p.const_i] = 0;
        for (int j = 0; j < D; j++) vout[j] = w.out[p.line[i]][j] - cen[j];
        orient(n, vout);
        for (int j = 0; j < D; j++) acc[i][j] = n[j];
    }
    for (int i = 0; i < p.nlines; i++)
        for (int j = 0; j < D; j++) normal[j] += acc[i][j];
}

/* Cube::split_to_squares + construct_polygons + check_ambiguous
 * (cornelius.cpp:1502-1650).  Returns the cube's number of lines; its
 * polygons are appended to w.poly, and *ambiguous reports the cube flag. */
static __device__ int cube_polygons(WorkRef &w, const double cube[2][2][2], int const_i, double const_v, double E0,
                             const double *dx, bool *ambiguous)
{
    int x1 = -1, x2 = -1, x3 = -1;
    for (int i = 0; i < D; i++)
        if (i != const_i) { if (x1 < 0) x1 = i; else if (x2 < 0) x2 = i; else x3 = i; }
    const int first = w.nl;
    int amb = 0;
    for (int i = 0; i < D; i++) {
        if (i == const_i) continue;
        for (int j = 0; j < 2; j++) {
            double sq[2][2];
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++)
                    sq[a][b] = (i == x1) ? cube[j][a][b] : (i == x2) ? cube[a][j][b] : cube[a][b][j];
            int before = w.nl;
            square_lines(w, sq, const_i, i, const_v, j * dx[i], E0, dx);
            if (w.nl - before == 2) amb++;   /* two lines <=> four cuts: Square::ambiguous */
            if (w.error) return 0;
        }
    }
    const int nlines = w.nl - first;
    *ambiguous = false;
    if (nlines == 0) return 0;
    if (amb == 0 && nlines == 6) amb++;
    *ambiguous = amb > 0;
    if (amb > 0) {
        bool not_used[12];
        int used = 0;
        for (int i = 0; i < nlines; i++) not_used[i] = true;
        do {
            if (nlines - used < 3 || w.np >= w.pcap) { w.error = true; return nlines; }
            Poly &p = w.poly[w.np];
            poly_init(p, const_i);
            for (int i = 0; i < nlines; i++)
                if (not_used[i] && poly_add_line(w, p, first + i, false)) { not_used[i] = false; used++; i = 0; }
            if (w.error) return nlines;
            w.np++;
        } while (used < nlines);
    } else {
        if (w.np >= w.pcap) { w.error = true; return nlines; }
        Poly &p = w.poly[w.np];
        poly_init(p, const_i);
        for (int i = 0; i < nlines; i++) poly_add_line(w, p, first + i, true);
        w.np++;
    }
    return nlines;
}

/* cube_polygons' line count and square ambiguity count (squares with two
 * lines) from the corner comparisons alone; err as square_lines would set
 * it.  cube_polygons then finds exactly this many lines. */
__device__ __forceinline__ int cube_line_count(const double cube[2][2][2], int const_i, double E0, int &amb, bool &err)
{
    int x1 = -1, x2 = -1;
    for (int i = 0; i < D; i++)
        if (i != const_i) { if (x1 < 0) x1 = i; else if (x2 < 0) x2 = i; }
    int n = 0;
    amb = 0;
    for (int i = 0; i < D; i++) {
        if (i == const_i) continue;
        for (int j = 0; j < 2; j++) {
            double sq[2][2];
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++)
                    sq[a][b] = (i == x1) ? cube[j][a][b] : (i == x2) ? cube[a][j][b] : cube[a][b][j];
            const int nc = square_cut_count(sq, E0);
            if (nc != 0 && nc != 2 && nc != 4) err = true;
            n += nc / 2;
            if (nc == 4) amb++;
        }
    }
    return n;
}

/* Cornelius::find_surface_3d for a cube whose corner (i,j,k) spans
 * (tau, x, y); dx3 = {dtau, dx, dy} (cornelius.cpp:2161-2237, init :2087).
 * Element geometry is 4-vectors with component 0 unused. */
static __device__ int surface_3d(Work &wk, const double cube[2][2][2], double E0, const double *dx3,
                          double cen[][D], double nor[][D])
{
    int above = 0;
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) for (int k = 0; k < 2; k++)
        if (cube[i][j][k] >= E0) above++;
    if (above == 0 || above == 8) return 0;
    const double dx[D] = {1, dx3[0], dx3[1], dx3[2]};
    WorkRef w = work_ref(wk);
    bool amb;
    cube_polygons(w, cube, 0, 0, E0, dx, &amb);
    if (w.error) return -1;
    if (w.np > kMaxElements) { w.error = true; return -1; }
    for (int i = 0; i < w.np; i++) {
        poly_normal(w, w.poly[i], nor[i]);
        const double *c = poly_centroid(w, w.poly[i]);
        for (int j = 0; j < D; j++) cen[i][j] = c[j];
    }
    return w.np;
}

/* Polyhedron::lines_equal, cornelius.cpp:786-802 */
__device__ __forceinline__ bool lines_equal(const WorkRef &w, int l1, int l2)
{
    const double *p11 = lstart(w, l1), *p12 = lend(w, l1), *p21 = lstart(w, l2);
    double diff1 = 0, diff2 = 0;
    for (int i = 0; i < D; i++) {
        diff1 += fabs(p11[i] - p21[i]);
        diff2 += fabs(p12[i] - p21[i]);
        if (diff1 > 1e-10 && diff2 > 1e-10) return false;
    }
    return true;
}

/* Polyhedron::tetravolume, cornelius.cpp:815-835 */
__device__ __forceinline__ void tetravolume(const double *a, const double *b, const double *c, double *n)
{
    double bc01 = b[0] * c[1] - b[1] * c[0];
    double bc02 = b[0] * c[2] - b[2] * c[0];
    double bc03 = b[0] * c[3] - b[3] * c[0];
    double bc12 = b[1] * c[2] - b[2] * c[1];
    double bc13 = b[1] * c[3] - b[3] * c[1];
    double bc23 = b[2] * c[3] - b[3] * c[2];
    n[0] = 1.0 / 6.0 * (a[1] * bc23 - a[2] * bc13 + a[3] * bc12);
    n[1] = -1.0 / 6.0 * (a[0] * bc23 - a[2] * bc03 + a[3] * bc02);
    n[2] = 1.0 / 6.0 * (a[0] * bc13 - a[1] * bc03 + a[3] * bc01);
    n[3] = -1.0 / 6.0 * (a[0] * bc12 - a[1] * bc02 + a[2] * bc01);
}

struct Hedron {
    unsigned char poly[24];
    int npoly, ntet;
};

/* Polyhedron::add_polygon, cornelius.cpp:743-774 */
__device__ __forceinline__ bool hedron_add(WorkRef &w, Hedron &h, int pi, bool donocheck)
{
    const Poly &p = w.poly[pi];
    if (donocheck || h.npoly == 0) {
        if (h.npoly >= 24) { w.error = true; return false; }
        h.poly[h.npoly++] = (unsigned char)pi;
        h.ntet += p.nlines;
        return true;
    }
    for (int i = 0; i < h.npoly; i++) {
        const Poly &q = w.poly[h.poly[i]];
        for (int j = 0; j < p.nlines; j++)
            for (int k = 0; k < q.nlines; k++)
                if (lines_equal(w, p.line[j], q.line[k])) {
                    if (h.npoly >= 24) { w.error = true; return false; }
                    h.poly[h.npoly++] = (unsigned char)pi;
                    h.ntet += p.nlines;
                    return true;
                }
    }
    return false;
}

/* Polyhedron::calculate_centroid and calculate_normal, cornelius.cpp:842-987 */
static __device__ void hedron_geometry(const WorkRef &w, const Hedron &h, double *centroid, double *normal)
{
    double mean[D] = {0, 0, 0, 0};
    for (int i = 0; i < h.npoly; i++) {
        const Poly &p = w.poly[h.poly[i]];
        for (int j = 0; j < p.nlines; j++) {
            const double *p1 = lstart(w, p.line[j]), *p2 = lend(w, p.line[j]);
            for (int k = 0; k < D; k++) mean[k] += p1[k] + p2[k];
        }
    }
    for (int j = 0; j < D; j++) mean[j] = mean[j] / (double)(2.0 * h.ntet);
    double up[D] = {0, 0, 0, 0}, down = 0;
    for (int i = 0; i < h.npoly; i++) {
        Poly &p = w.poly[h.poly[i]];
        const double *cent = poly_centroid(w, p);
        for (int j = 0; j < p.nlines; j++) {
            const double *p1 = lstart(w, p.line[j]), *p2 = lend(w, p.line[j]);
            double cm[D], a[D], b[D], c[D], n[D];
            for (int k = 0; k < D; k++) cm[k] = (p1[k] + p2[k] + cent[k] + mean[k]) / 4.0;
            for (int k = 0; k < D; k++) { a[k] = p1[k] - mean[k]; b[k] = p2[k] - mean[k]; c[k] = cent[k] - mean[k]; }
            tetravolume(a, b, c, n);
            double V = 0;
            for (int k = 0; k < D; k++) V += n[k] * n[k];
            V = sqrt(V);
            for (int k = 0; k < D; k++) up[k] += cm[k] * V;
            down += V;
        }
    }
    for (int i = 0; i < D; i++) centroid[i] = up[i] / down;
    for (int i = 0; i < D; i++) normal[i] = 0;
    /* the reference sums the oriented tetrahedron normals after computing all
     * of them; the same order of additions is kept here */
    for (int i = 0; i < h.npoly; i++) {
        Poly &p = w.poly[h.poly[i]];
        const double *cent = poly_centroid(w, p);
        for (int j = 0; j < p.nlines; j++) {
            const double *p1 = lstart(w, p.line[j]), *p2 = lend(w, p.line[j]);
            double a[D], b[D], c[D], n[D], vout[D];
            for (int k = 0; k < D; k++) { a[k] = p1[k] - centroid[k]; b[k] = p2[k] - centroid[k]; c[k] = cent[k] - centroid[k]; }
            tetravolume(a, b, c, n);
            for (int k = 0; k < D; k++) vout[k] = w.out[p.line[j]][k] - centroid[k];
            orient(n, vout);
            for (int k = 0; k < D; k++) normal[k] += n[k];
        }
    }
}

/* Cornelius::find_surface_4d with the Hypercube construction
 * (cornelius.cpp:1778-1970, :2248-2287). */
static __device__ int surface_4d(Work &wk, const double h[2][2][2][2], double E0, const double *dx,
                          double cen[][D], double nor[][D])
{
    int above = 0;
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) for (int k = 0; k < 2; k++) for (int l = 0; l < 2; l++)
        if (h[i][j][k][l] >= E0) above++;
    if (above == 0 || above == 16) return 0;
    WorkRef w = work_ref(wk);
    int nlines_total = 0, ambiguous = 0;
    for (int i = 0; i < D; i++)
        for (int j = 0; j < 2; j++) {
            double cu[2][2][2];
            for (int a = 0; a < 2; a++) for (int b = 0; b < 2; b++) for (int c = 0; c < 2; c++)
                cu[a][b][c] = (i == 0) ? h[j][a][b][c] : (i == 1) ? h[a][j][b][c] : (i == 2) ? h[a][b][j][c] : h[a][b][c][j];
            bool amb;
            nlines_total += cube_polygons(w, cu, i, j * dx[i], E0, dx, &amb);
            if (w.error) return -1;
            if (amb) ambiguous++;
        }
    if (ambiguous == 0) {
        int points = 0;
        for (int a = 0; a < 2; a++) for (int b = 0; b < 2; b++) for (int c = 0; c < 2; c++) for (int d = 0; d < 2; d++)
            if (h[a][b][c][d] < E0) points++;
        if (points > 8) points = 16 - points;
        if (nlines_total == 24 && points == 2) ambiguous++;
    }
    Hedron hed[kMaxHedra];
    int nh = 0;
    const int npolys = w.np;
    if (ambiguous > 0) {
        bool not_used[kMaxPoly];
        int used = 0;
        for (int i = 0; i < npolys; i++) not_used[i] = true;
        do {
            if (nh >= kMaxHedra) { w.error = true; return -1; }
            hed[nh].npoly = 0; hed[nh].ntet = 0;
            for (int i = 0; i < npolys; i++)
                if (not_used[i] && hedron_add(w, hed[nh], i, false)) { not_used[i] = false; used++; i = 0; }
            if (w.error) return -1;
            nh++;
        } while (used < npolys);
    } else {
        hed[0].npoly = 0; hed[0].ntet = 0;
        for (int i = 0; i < npolys; i++) hedron_add(w, hed[0], i, true);
        if (w.error) return -1;
        nh = 1;
    }
    for (int i = 0; i < nh; i++) hedron_geometry(w, hed[i], cen[i], nor[i]);
    return nh;
}

} // namespace cor
} // namespace vh

#endif
