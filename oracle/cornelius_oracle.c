/*
 * cornelius_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of the
 * Cornelius 1.3 iso-surface finder (P. Huovinen and H. Petersen,
 * arXiv:1206.3371; vendored by the reference as
 * freezeout/cornelius-c++-1.3/cornelius.cpp) and of the reference's freezeout
 * driver (freezeout/FreezeOut.cpp), for the 3D (2+1D hydro) and 4D (3+1D
 * hydro) cases the hot path uses.  Plain C with fixed-size storage; the
 * operation order of every floating-point expression follows the reference.
 *
 * Pinned by tests/test_oracle_vs_reference.py against the reference's own
 * known-answer files output_3d.dat / output_4d.dat (example_cornelius.cpp:
 * 10^4 glibc rand() cubes and hypercubes, threshold 0.5; hashes in
 * tests/golden/cornelius_kat.json) and against the reference's freezeout
 * output for whole hydro runs.
 *
 * MODIFIED VERSION of the Cornelius subroutine: restated in 2026 in plain C
 * (fixed-size storage, status codes instead of exit()), with the same
 * arithmetic.  The original copyright and permission notice follows; this
 * file is distributed under the same terms.
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
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define DIM 4

typedef struct {
    double corners[2][DIM];
    double out[DIM];
    int start, end;
} Line;

typedef struct {
    Line *lines[24];
    int nlines, const_i, x1, x2, x3;
    double centroid[DIM], normal[DIM];
    int have_centroid;
} Polygon;

typedef struct {
    Polygon *polys[24];
    int npoly, ntet;
    double centroid[DIM], normal[DIM];
} Polyhedron;

typedef struct {
    double points[2][2];
    double cuts[4][2], out[4][2];
    int const_i[2];
    double const_v[2];
    int x1, x2, ncuts, nlines, ambiguous;
    Line lines[2];
} Square;

typedef struct {
    double cube[2][2][2];
    Square squares[6];
    Line *lines[12];
    Polygon polys[8];
    int nlines, npoly, ambiguous, const_i, x1, x2, x3;
    double const_v;
} Cube;

static int g_error;  /* set where the reference prints an error and exit(1)s */

static double *line_start(Line *l) { return l->corners[l->start]; }
static double *line_end(Line *l) { return l->corners[l->end]; }

/* cornelius.cpp:91-106 */
static void check_normal_direction(double *n, const double *out)
{
    double dot = 0;
    for (int i = 0; i < DIM; i++) dot += out[i] * n[i];
    if (dot < 0)
        for (int i = 0; i < DIM; i++) n[i] = -n[i];
}

/* ------------------------------------------------------------ Polygon */
static void polygon_init(Polygon *p, int c)
{
    p->const_i = c;
    p->x1 = p->x2 = p->x3 = -1;
    for (int i = 0; i < DIM; i++)
        if (i != c) {
            if (p->x1 < 0) p->x1 = i;
            else if (p->x2 < 0) p->x2 = i;
            else p->x3 = i;
        }
    p->nlines = 0;
    p->have_centroid = 0;
}

/* cornelius.cpp:436-471 */
static int polygon_add_line(Polygon *p, Line *l, int donotcheck)
{
    const double eps = 1e-10;
    if (donotcheck || p->nlines == 0) { p->lines[p->nlines++] = l; return 1; }
    double *p1 = line_start(l), *p2 = line_end(l), *p3 = line_end(p->lines[p->nlines - 1]);
    double diff1 = 0, diff2 = 0;
    for (int j = 0; j < DIM; j++) { diff1 += fabs(p1[j] - p3[j]); diff2 += fabs(p2[j] - p3[j]); }
    if (diff1 < eps || diff2 < eps) {
        if (diff2 < eps) { int t = l->start; l->start = l->end; l->end = t; }
        p->lines[p->nlines++] = l;
        return 1;
    }
    return 0;
}

/* cornelius.cpp:478-551 */
static double *polygon_centroid(Polygon *p)
{
    if (p->have_centroid) return p->centroid;
    double mean[DIM] = {0, 0, 0, 0};
    for (int i = 0; i < p->nlines; i++) {
        double *p1 = line_start(p->lines[i]), *p2 = line_end(p->lines[i]);
        for (int j = 0; j < DIM; j++) mean[j] += p1[j] + p2[j];
    }
    for (int j = 0; j < DIM; j++) mean[j] = mean[j] / (double)(2.0 * p->nlines);
    if (p->nlines == 3) {
        for (int i = 0; i < DIM; i++) p->centroid[i] = mean[i];
        p->have_centroid = 1;
        return p->centroid;
    }
    double sum_up[DIM] = {0, 0, 0, 0}, sum_down = 0, a[DIM], b[DIM], cm[DIM];
    const int x1 = p->x1, x2 = p->x2, x3 = p->x3;
    for (int i = 0; i < p->nlines; i++) {
        double *p1 = line_start(p->lines[i]), *p2 = line_end(p->lines[i]);
        for (int j = 0; j < DIM; j++) cm[j] = (p1[j] + p2[j] + mean[j]) / 3.0;
        for (int j = 0; j < DIM; j++) { a[j] = p1[j] - mean[j]; b[j] = p2[j] - mean[j]; }
        double A_i = 0.5 * sqrt(pow(a[x2] * b[x3] - a[x3] * b[x2], 2.0) + pow(a[x1] * b[x3] - a[x3] * b[x1], 2.0) +
                                pow(a[x2] * b[x1] - a[x1] * b[x2], 2.0));
        for (int j = 0; j < DIM; j++) sum_up[j] += cm[j] * A_i;
        sum_down += A_i;
    }
    for (int i = 0; i < DIM; i++) p->centroid[i] = sum_up[i] / sum_down;
    p->have_centroid = 1;
    return p->centroid;
}

/* cornelius.cpp:559-617 */
static void polygon_normal(Polygon *p, double *normal)
{
    double *cen = polygon_centroid(p);
    double a[DIM], b[DIM], n[DIM], Vout[DIM];
    for (int i = 0; i < DIM; i++) normal[i] = 0;
    double acc[24][DIM];
    for (int i = 0; i < p->nlines; i++) {
        double *p1 = line_start(p->lines[i]), *p2 = line_end(p->lines[i]);
        for (int j = 0; j < DIM; j++) { a[j] = p1[j] - cen[j]; b[j] = p2[j] - cen[j]; }
        for (int j = 0; j < DIM; j++) n[j] = 0;
        n[p->x1] = 0.5 * (a[p->x2] * b[p->x3] - a[p->x3] * b[p->x2]);
        n[p->x2] = -0.5 * (a[p->x1] * b[p->x3] - a[p->x3] * b[p->x1]);
        n[p->x3] = 0.5 * (a[p->x1] * b[p->x2] - a[p->x2] * b[p->x1]);
        n[p->const_i] = 0;
        double *o = p->lines[i]->out;
        for (int j = 0; j < DIM; j++) Vout[j] = o[j] - cen[j];
        check_normal_direction(n, Vout);
        for (int j = 0; j < DIM; j++) acc[i][j] = n[j];
    }
    for (int i = 0; i < p->nlines; i++)
        for (int j = 0; j < DIM; j++) normal[j] += acc[i][j];
}

/* --------------------------------------------------------- Polyhedron */
/* cornelius.cpp:786-802 */
static int lines_equal(Line *l1, Line *l2)
{
    const double eps = 1e-10;
    double *p11 = line_start(l1), *p12 = line_end(l1), *p21 = line_start(l2);
    double diff1 = 0, diff2 = 0;
    for (int i = 0; i < DIM; i++) {
        diff1 += fabs(p11[i] - p21[i]);
        diff2 += fabs(p12[i] - p21[i]);
        if (diff1 > eps && diff2 > eps) return 0;
    }
    return 1;
}

/* cornelius.cpp:743-774 */
static int polyhedron_add(Polyhedron *h, Polygon *p, int donocheck)
{
    if (donocheck || h->npoly == 0) {
        h->polys[h->npoly++] = p;
        h->ntet += p->nlines;
        return 1;
    }
    for (int i = 0; i < h->npoly; i++)
        for (int j = 0; j < p->nlines; j++)
            for (int k = 0; k < h->polys[i]->nlines; k++)
                if (lines_equal(p->lines[j], h->polys[i]->lines[k])) {
                    h->polys[h->npoly++] = p;
                    h->ntet += p->nlines;
                    return 1;
                }
    return 0;
}

/* cornelius.cpp:815-835 */
static void tetravolume(const double *a, const double *b, const double *c, double *n)
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

/* cornelius.cpp:842-920 */
static void polyhedron_centroid(Polyhedron *h)
{
    double mean[DIM] = {0, 0, 0, 0};
    for (int i = 0; i < h->npoly; i++)
        for (int j = 0; j < h->polys[i]->nlines; j++) {
            double *p1 = line_start(h->polys[i]->lines[j]), *p2 = line_end(h->polys[i]->lines[j]);
            for (int k = 0; k < DIM; k++) mean[k] += p1[k] + p2[k];
        }
    for (int j = 0; j < DIM; j++) mean[j] = mean[j] / (double)(2.0 * h->ntet);
    double a[DIM], b[DIM], c[DIM], n[DIM], cm[DIM], sum_up[DIM] = {0, 0, 0, 0}, sum_down = 0;
    for (int i = 0; i < h->npoly; i++) {
        double *cent = polygon_centroid(h->polys[i]);
        for (int j = 0; j < h->polys[i]->nlines; j++) {
            double *p1 = line_start(h->polys[i]->lines[j]), *p2 = line_end(h->polys[i]->lines[j]);
            for (int k = 0; k < DIM; k++) cm[k] = (p1[k] + p2[k] + cent[k] + mean[k]) / 4.0;
            for (int k = 0; k < DIM; k++) { a[k] = p1[k] - mean[k]; b[k] = p2[k] - mean[k]; c[k] = cent[k] - mean[k]; }
            tetravolume(a, b, c, n);
            double V = 0;
            for (int k = 0; k < DIM; k++) V += n[k] * n[k];
            V = sqrt(V);
            for (int k = 0; k < DIM; k++) sum_up[k] += cm[k] * V;
            sum_down += V;
        }
    }
    for (int i = 0; i < DIM; i++) h->centroid[i] = sum_up[i] / sum_down;
}

/* cornelius.cpp:928-987 */
static void polyhedron_normal(Polyhedron *h)
{
    double a[DIM], b[DIM], c[DIM], Vout[DIM], nn[96][DIM];
    int nt = 0;
    for (int i = 0; i < h->npoly; i++) {
        double *cent = polygon_centroid(h->polys[i]);
        for (int j = 0; j < h->polys[i]->nlines; j++) {
            Line *l = h->polys[i]->lines[j];
            double *p1 = line_start(l), *p2 = line_end(l);
            for (int k = 0; k < DIM; k++) { a[k] = p1[k] - h->centroid[k]; b[k] = p2[k] - h->centroid[k]; c[k] = cent[k] - h->centroid[k]; }
            tetravolume(a, b, c, nn[nt]);
            for (int k = 0; k < DIM; k++) Vout[k] = l->out[k] - h->centroid[k];
            check_normal_direction(nn[nt], Vout);
            nt++;
        }
    }
    for (int i = 0; i < DIM; i++) h->normal[i] = 0;
    for (int i = 0; i < nt; i++)
        for (int j = 0; j < DIM; j++) h->normal[j] += nn[i][j];
}

/* ------------------------------------------------------------- Square */
static void square_init(Square *q, double sq[2][2], const int *c_i, const double *c_v)
{
    memcpy(q->points, sq, sizeof(q->points));
    q->const_i[0] = c_i[0]; q->const_i[1] = c_i[1];
    q->const_v[0] = c_v[0]; q->const_v[1] = c_v[1];
    q->x1 = q->x2 = -1;
    for (int i = 0; i < DIM; i++)
        if (i != c_i[0] && i != c_i[1]) {
            if (q->x1 < 0) q->x1 = i; else q->x2 = i;
        }
    q->ncuts = q->nlines = q->ambiguous = 0;
}

/* cornelius.cpp:1192-1254 */
static void ends_of_edge(Square *q, double E0, const double *dx)
{
    double (*P)[2] = q->points;
    double (*C)[2] = q->cuts;
    const double d1 = dx[q->x1], d2 = dx[q->x2];
#define CUT(a, b) do { C[q->ncuts][0] = (a); C[q->ncuts][1] = (b); q->ncuts++; } while (0)
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
    if (q->ncuts != 0 && q->ncuts != 2 && q->ncuts != 4) g_error = 1;
}

/* cornelius.cpp:1263-1337 */
static void find_outside(Square *q, double E0, const double *dx)
{
    double (*P)[2] = q->points;
    const double d1 = dx[q->x1], d2 = dx[q->x2];
    if (q->ncuts == 4) {
        q->ambiguous = 1;
        double Emid = 0;
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) Emid += 0.25 * P[i][j];
        if ((P[0][0] < E0 && Emid < E0) || (P[0][0] > E0 && Emid > E0))
            for (int i = 0; i < 2; i++) { double t = q->cuts[1][i]; q->cuts[1][i] = q->cuts[2][i]; q->cuts[2][i] = t; }
        if ((Emid - E0) < 0) {
            for (int i = 0; i < 2; i++) { q->out[i][0] = 0.5 * d1; q->out[i][1] = 0.5 * d2; }
        } else if ((P[0][0] - E0) < 0) {
            q->out[0][0] = 0; q->out[0][1] = 0; q->out[1][0] = d1; q->out[1][1] = d2;
        } else {
            q->out[0][0] = d1; q->out[0][1] = 0; q->out[1][0] = 0; q->out[1][1] = d2;
        }
    } else {
        for (int i = 0; i < 2; i++) { q->out[i][0] = 0; q->out[i][1] = 0; }
        int nout = 0;
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++)
                if (P[i][j] < E0) { q->out[0][0] += i * d1; q->out[0][1] += j * d2; nout++; }
        if (nout > 0)
            for (int i = 0; i < 2; i++)
                for (int j = 0; j < 2; j++) q->out[i][j] = q->out[i][j] / (double)nout;
    }
}

/* cornelius.cpp:1134-1173 and Line::init (:208-251) */
static void square_lines(Square *q, double E0, const double *dx)
{
    int above = 0;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            if (q->points[i][j] >= E0) above++;
    if (above == 0 || above == 4) { q->nlines = 0; return; }
    ends_of_edge(q, E0, dx);
    if (q->ncuts > 0) find_outside(q, E0, dx);
    double pt[2][DIM], out[DIM];
    for (int i = 0; i < q->ncuts; i++) {
        pt[i % 2][q->x1] = q->cuts[i][0];
        pt[i % 2][q->x2] = q->cuts[i][1];
        pt[i % 2][q->const_i[0]] = q->const_v[0];
        pt[i % 2][q->const_i[1]] = q->const_v[1];
        if (i % 2 == 1) {
            out[q->x1] = q->out[i / 2][0];
            out[q->x2] = q->out[i / 2][1];
            out[q->const_i[0]] = q->const_v[0];
            out[q->const_i[1]] = q->const_v[1];
            Line *l = &q->lines[i / 2];
            memcpy(l->corners, pt, sizeof(pt));
            memcpy(l->out, out, sizeof(out));
            l->start = 0; l->end = 1;
            q->nlines++;
        }
    }
}

/* --------------------------------------------------------------- Cube */
static void cube_init(Cube *c, double cu[2][2][2], int c_i, double c_v)
{
    c->const_i = c_i; c->const_v = c_v;
    c->x1 = c->x2 = c->x3 = -1;
    for (int i = 0; i < DIM; i++)
        if (i != c_i) {
            if (c->x1 < 0) c->x1 = i; else if (c->x2 < 0) c->x2 = i; else c->x3 = i;
        }
    memcpy(c->cube, cu, sizeof(c->cube));
    c->nlines = c->npoly = c->ambiguous = 0;
}

/* cornelius.cpp:1502-1542 */
static void split_to_squares(Cube *c, const double *dx)
{
    int n = 0;
    double sq[2][2];
    int ci[2];
    double cv[2];
    for (int i = 0; i < DIM; i++) {
        if (i == c->const_i) continue;
        ci[0] = c->const_i; ci[1] = i;
        for (int j = 0; j < 2; j++) {
            cv[0] = c->const_v; cv[1] = j * dx[i];
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++)
                    sq[a][b] = (i == c->x1) ? c->cube[j][a][b] : (i == c->x2) ? c->cube[a][j][b] : c->cube[a][b][j];
            square_init(&c->squares[n], sq, ci, cv);
            n++;
        }
    }
}

/* cornelius.cpp:1552-1650 */
static void cube_polygons(Cube *c, double v0, const double *dx)
{
    split_to_squares(c, dx);
    for (int i = 0; i < 6; i++) square_lines(&c->squares[i], v0, dx);
    c->nlines = 0;
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < c->squares[i].nlines; j++) c->lines[c->nlines++] = &c->squares[i].lines[j];
    if (c->nlines == 0) return;
    for (int i = 0; i < 6; i++) if (c->squares[i].ambiguous) c->ambiguous++;
    if (c->ambiguous == 0 && c->nlines == 6) c->ambiguous++;
    if (c->ambiguous > 0) {
        int not_used[12], used = 0;
        for (int i = 0; i < c->nlines; i++) not_used[i] = 1;
        do {
            if (c->nlines - used < 3 || c->npoly >= 8) { g_error = 1; return; }
            polygon_init(&c->polys[c->npoly], c->const_i);
            for (int i = 0; i < c->nlines; i++)
                if (not_used[i] && polygon_add_line(&c->polys[c->npoly], c->lines[i], 0)) {
                    not_used[i] = 0;
                    used++;
                    i = 0;
                }
            c->npoly++;
        } while (used < c->nlines);
    } else {
        polygon_init(&c->polys[0], c->const_i);
        for (int i = 0; i < c->nlines; i++) polygon_add_line(&c->polys[0], c->lines[i], 1);
        c->npoly = 1;
    }
}

/* ------------------------------------------------------------ drivers */
/* Cornelius::find_surface_3d (cornelius.cpp:2161-2237) with init(3, v0, dx3)
 * (:2087-2102): writes up to 8 elements as 4-vectors (index 0 unused). */
static int surface_3d(const double cube[2][2][2], double v0, const double *dx3, double cen[][DIM], double nor[][DIM])
{
    int above = 0;
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) for (int k = 0; k < 2; k++)
        if (cube[i][j][k] >= v0) above++;
    if (above == 0 || above == 8) return 0;
    double dx[DIM] = {1, dx3[0], dx3[1], dx3[2]};
    static __thread Cube c;
    double cu[2][2][2];
    memcpy(cu, cube, sizeof(cu));
    cube_init(&c, cu, 0, 0);
    cube_polygons(&c, v0, dx);
    for (int i = 0; i < c.npoly; i++) {
        polygon_normal(&c.polys[i], nor[i]);
        double *cc = polygon_centroid(&c.polys[i]);
        for (int j = 0; j < DIM; j++) cen[i][j] = cc[j];
    }
    return c.npoly;
}

/* Cornelius::find_surface_4d (cornelius.cpp:2248-2287), Hypercube
 * (:1778-1970). */
static int surface_4d(const double h[2][2][2][2], double v0, const double *dx, double cen[][DIM], double nor[][DIM])
{
    int above = 0;
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) for (int k = 0; k < 2; k++) for (int l = 0; l < 2; l++)
        if (h[i][j][k][l] >= v0) above++;
    if (above == 0 || above == 16) return 0;
    static __thread Cube cubes[8];
    static __thread Polyhedron hedra[10];
    Polygon *polys[80];
    int npolys = 0, nc = 0;
    double cu[2][2][2];
    for (int i = 0; i < DIM; i++)
        for (int j = 0; j < 2; j++) {
            double cv = j * dx[i];
            for (int a = 0; a < 2; a++) for (int b = 0; b < 2; b++) for (int c = 0; c < 2; c++)
                cu[a][b][c] = (i == 0) ? h[j][a][b][c] : (i == 1) ? h[a][j][b][c] : (i == 2) ? h[a][b][j][c] : h[a][b][c][j];
            cube_init(&cubes[nc], cu, i, cv);
            nc++;
        }
    for (int i = 0; i < 8; i++) cube_polygons(&cubes[i], v0, dx);
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < cubes[i].npoly; j++) polys[npolys++] = &cubes[i].polys[j];
    int ambiguous = 0;
    for (int i = 0; i < 8; i++) if (cubes[i].ambiguous) ambiguous++;
    if (ambiguous == 0) {
        int nlines = 0, points = 0;
        for (int i = 0; i < 8; i++) nlines += cubes[i].nlines;
        for (int a = 0; a < 2; a++) for (int b = 0; b < 2; b++) for (int c = 0; c < 2; c++) for (int d = 0; d < 2; d++)
            if (h[a][b][c][d] < v0) points++;
        if (points > 8) points = 16 - points;
        if (nlines == 24 && points == 2) ambiguous++;
    }
    int nh = 0;
    if (ambiguous > 0) {
        int not_used[80], used = 0;
        for (int i = 0; i < npolys; i++) not_used[i] = 1;
        do {
            if (nh >= 10) { g_error = 1; return 0; }
            hedra[nh].npoly = 0; hedra[nh].ntet = 0;
            for (int i = 0; i < npolys; i++)
                if (not_used[i] && polyhedron_add(&hedra[nh], polys[i], 0)) { not_used[i] = 0; used++; i = 0; }
            nh++;
        } while (used < npolys);
    } else {
        hedra[0].npoly = 0; hedra[0].ntet = 0;
        for (int i = 0; i < npolys; i++) polyhedron_add(&hedra[0], polys[i], 1);
        nh = 1;
    }
    for (int i = 0; i < nh; i++) {
        polyhedron_centroid(&hedra[i]);
        polyhedron_normal(&hedra[i]);
        for (int j = 0; j < DIM; j++) { cen[i][j] = hedra[i].centroid[j]; nor[i][j] = hedra[i].normal[j]; }
    }
    return nh;
}

/* Batch entry for the known-answer tests: cubes (8 values) or hypercubes (16)
 * in C order; writes per element (2*dim doubles: centroid then normal, the
 * dim trailing components as get_centroid_elem/get_normal_elem return them)
 * and the element count of every cube.  Returns the total or -1 on error. */
int vho_cornelius_batch(int dim, const double *cubes, int n, double v0, const double *dx,
                        double *out, int cap, int *counts)
{
    int total = 0;
    g_error = 0;
    double cen[10][DIM], nor[10][DIM];
    for (int c = 0; c < n; c++) {
        int ne;
        if (dim == 3) ne = surface_3d((const double(*)[2][2])(cubes + 8 * (size_t)c), v0, dx, cen, nor);
        else ne = surface_4d((const double(*)[2][2][2])(cubes + 16 * (size_t)c), v0, dx, cen, nor);
        if (g_error) return -1;
        counts[c] = ne;
        for (int e = 0; e < ne; e++) {
            if (total >= cap) return -1;
            for (int j = 0; j < dim; j++) out[(size_t)total * 2 * dim + j] = cen[e][j + DIM - dim];
            for (int j = 0; j < dim; j++) out[(size_t)total * 2 * dim + dim + j] = nor[e][j + DIM - dim];
            total++;
        }
    }
    return total;
}

/* ---------------------------------------------------- freezeout driver */
/* The oracle state lives in vh_oracle.c; it exposes what this file needs. */
typedef struct vho_t vho_t;
int vho_fo_view(vho_t *h, int *dims, double *spacing, double *t0dt_t, int *n_next, double **e, double **u,
                double **q, int *nq, double **slabs_prev, double **slabs_cur, double *eF);
double vho_T_of_e(vho_t *h, double ed);
double vho_p_of_e(vho_t *h, double ed);
void vho_fo_flip(vho_t *h);

/* FreezeOut.cpp:40-55 */
static double interp3(double x0, double x1, double x2, double a000, double a100, double a010, double a001,
                      double a110, double a101, double a011, double a111)
{
    return ((1 - x0) * (1 - x1) * (1 - x2) * a000) + ((x0) * (1 - x1) * (1 - x2) * a100) + ((1 - x0) * (x1) * (1 - x2) * a010) +
           ((1 - x0) * (1 - x1) * (x2) * a001) + ((x0) * (x1) * (1 - x2) * a110) + ((x0) * (1 - x1) * (x2) * a101) +
           ((1 - x0) * (x1) * (x2) * a011) + ((x0) * (x1) * (x2) * a111);
}

/* FreezeOut.cpp:13-38 (note the a1011 term precedes a0111 in the sum) */
static double interp4(double x0, double x1, double x2, double x3,
                      double a0000, double a1000, double a0100, double a0010, double a0001,
                      double a1100, double a1010, double a1001, double a0110, double a0101, double a0011,
                      double a1110, double a1101, double a0111, double a1011, double a1111)
{
    return ((1 - x0) * (1 - x1) * (1 - x2) * (1 - x3) * a0000) + ((x0) * (1 - x1) * (1 - x2) * (1 - x3) * a1000) +
           ((1 - x0) * (x1) * (1 - x2) * (1 - x3) * a0100) + ((1 - x0) * (1 - x1) * (x2) * (1 - x3) * a0010) +
           ((1 - x0) * (1 - x1) * (1 - x2) * (x3) * a0001) + ((x0) * (x1) * (1 - x2) * (1 - x3) * a1100) +
           ((x0) * (1 - x1) * (x2) * (1 - x3) * a1010) + ((x0) * (1 - x1) * (1 - x2) * (x3) * a1001) +
           ((1 - x0) * (x1) * (x2) * (1 - x3) * a0110) + ((1 - x0) * (x1) * (1 - x2) * (x3) * a0101) +
           ((1 - x0) * (1 - x1) * (x2) * (x3) * a0011) + ((x0) * (x1) * (x2) * (1 - x3) * a1110) +
           ((x0) * (x1) * (1 - x2) * (x3) * a1101) + ((x0) * (1 - x1) * (x2) * (x3) * a1011) +
           ((1 - x0) * (x1) * (x2) * (x3) * a0111) + ((x0) * (x1) * (x2) * (x3) * a1111);
}

/* One freezeout block: swapAndSetHydroVariables (FreezeOut.cpp:57-97), the
 * finder (callFOFinder2p1D :282-361 or callFOFinder3p1D :200-280) and
 * checkForCellsAboveTc (:364-381).  Slab layout: [11][N], N = nx*ny*nz,
 * index ix + nx*(iy + ny*iz): e, then ux uy un e pixx pixy pixn piyy piyn Pi. */
int vho_freezeout(vho_t *h, double *out, int cap, int *n_el, int *n_above)
{
    int dims[3], n, nq;
    double sp[4], tt[3], *e, *u, *q, *prev, *cur, eF;
    vho_fo_view(h, dims, sp, tt, &n, &e, &u, &q, &nq, &prev, &cur, &eF);
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    const int ncx = nx + 4, ncy = ny + 4, ncz = nz + 4;
    const size_t N = (size_t)nx * ny * nz, L = (size_t)ncx * ncy * ncz;
    const double dx = sp[1], dy = sp[2], dz = sp[3], t0 = tt[0], dt = tt[1], t = tt[2];
    /* the caller flipped the slabs: prev holds the last block's values */
    int above = 0;
    for (int iz = 0; iz < nz; iz++)
        for (int iy = 0; iy < ny; iy++)
            for (int ix = 0; ix < nx; ix++) {
                size_t s = (ix + 2) + (size_t)ncx * ((iy + 2) + (size_t)ncy * (iz + 2));
                size_t m = ix + (size_t)nx * (iy + (size_t)ny * iz);
                cur[0 * N + m] = e[s];
                cur[1 * N + m] = u[1 * L + s];
                cur[2 * N + m] = u[2 * L + s];
                cur[3 * N + m] = u[3 * L + s];
                cur[4 * N + m] = e[s];
                cur[5 * N + m] = q[8 * L + s];
                cur[6 * N + m] = q[9 * L + s];
                cur[7 * N + m] = q[10 * L + s];
                cur[8 * N + m] = q[11 * L + s];
                cur[9 * N + m] = q[12 * L + s];
                cur[10 * N + m] = (nq == 15) ? q[14 * L + s] : 0.0;
                if (e[s] > eF) above++;
            }
    const int dim = (nz > 1) ? 4 : 3;
    double cen[10][DIM], nor[10][DIM];
    int total = 0;
    g_error = 0;
#define SL(slab, v, ix, iy, iz) ((slab) ? cur : prev)[(size_t)(v) * N + (ix) + (size_t)nx * ((iy) + (size_t)ny * (iz))]
    for (int ix = 0; ix < nx - 1; ix++)
        for (int iy = 0; iy < ny - 1; iy++)
            for (int iz = 0; iz < (dim == 4 ? nz - 1 : 1); iz++) {
                int ne;
                if (dim == 3) {
                    double cb[2][2][2];
                    for (int a = 0; a < 2; a++) for (int b = 0; b < 2; b++) for (int c = 0; c < 2; c++)
                        cb[a][b][c] = SL(a, 0, ix + b, iy + c, 0);
                    double dx3[3] = {sp[0], dx, dy};
                    ne = surface_3d(cb, eF, dx3, cen, nor);
                } else {
                    double hc[2][2][2][2];
                    for (int a = 0; a < 2; a++) for (int b = 0; b < 2; b++) for (int c = 0; c < 2; c++) for (int d = 0; d < 2; d++)
                        hc[a][b][c][d] = SL(a, 0, ix + b, iy + c, iz + d);
                    ne = surface_4d(hc, eF, sp, cen, nor);
                }
                if (g_error) return -2;
                for (int i = 0; i < ne; i++) {
                    if (total >= cap) return -1;
                    double *o = out + (size_t)total * 20;
                    double cell_tau = t0 + ((double)n) * dt;
                    double cell_x = (double)ix * dx - (((double)(nx - 1)) / 2.0 * dx);
                    double cell_y = (double)iy * dy - (((double)(ny - 1)) / 2.0 * dy);
                    double cell_z = (dim == 4) ? (double)iz * dz - (((double)(nz - 1)) / 2.0 * dz) : 0.0;
                    double tau_frac = cen[i][0] / sp[0];
                    double x_frac = cen[i][1] / dx;
                    double y_frac = cen[i][2] / dy;
                    double z_frac = (dim == 4) ? cen[i][3] / dz : 0.0;
                    /* in 3D the elements live in components 1..3 of the 4-vector */
                    if (dim == 3) { tau_frac = cen[i][1] / sp[0]; x_frac = cen[i][2] / dx; y_frac = cen[i][3] / dy; }
                    double vals[10];
                    for (int v = 0; v < 10; v++) {
                        int iv = v + 1;
                        if (dim == 3)
                            vals[v] = interp3(tau_frac, x_frac, y_frac,
                                              SL(0, iv, ix, iy, 0), SL(1, iv, ix, iy, 0), SL(0, iv, ix + 1, iy, 0), SL(0, iv, ix, iy + 1, 0),
                                              SL(1, iv, ix + 1, iy, 0), SL(1, iv, ix, iy + 1, 0), SL(0, iv, ix + 1, iy + 1, 0),
                                              SL(1, iv, ix + 1, iy + 1, 0));
                        else
                            vals[v] = interp4(tau_frac, x_frac, y_frac, z_frac,
                                              SL(0, iv, ix, iy, iz), SL(1, iv, ix, iy, iz), SL(0, iv, ix + 1, iy, iz),
                                              SL(0, iv, ix, iy + 1, iz), SL(0, iv, ix, iy, iz + 1), SL(1, iv, ix + 1, iy, iz),
                                              SL(1, iv, ix, iy + 1, iz), SL(1, iv, ix, iy, iz + 1), SL(0, iv, ix + 1, iy + 1, iz),
                                              SL(0, iv, ix + 1, iy, iz + 1), SL(0, iv, ix, iy + 1, iz + 1), SL(1, iv, ix + 1, iy + 1, iz),
                                              SL(1, iv, ix + 1, iy, iz + 1), SL(0, iv, ix + 1, iy + 1, iz + 1),
                                              SL(1, iv, ix, iy + 1, iz + 1), SL(1, iv, ix + 1, iy + 1, iz + 1));
                    }
                    if (dim == 3) {
                        o[0] = cen[i][1] + cell_tau; o[1] = cen[i][2] + cell_x; o[2] = cen[i][3] + cell_y; o[3] = 0.0;
                        o[4] = t * nor[i][1]; o[5] = t * nor[i][2]; o[6] = t * nor[i][3]; o[7] = 0.0;
                    } else {
                        o[0] = cen[i][0] + cell_tau; o[1] = cen[i][1] + cell_x; o[2] = cen[i][2] + cell_y; o[3] = cen[i][3] + cell_z;
                        o[4] = t * nor[i][0]; o[5] = t * nor[i][1]; o[6] = t * nor[i][2]; o[7] = t * nor[i][3];
                    }
                    o[8] = vals[0]; o[9] = vals[1]; o[10] = vals[2];
                    double eps = vals[3];
                    o[11] = eps;
                    o[12] = vho_T_of_e(h, eps);
                    o[13] = vho_p_of_e(h, eps);
                    o[14] = vals[4]; o[15] = vals[5]; o[16] = vals[6]; o[17] = vals[7]; o[18] = vals[8];
                    o[19] = vals[9];
                    total++;
                }
            }
#undef SL
    vho_fo_flip(h);
    *n_el = total;
    *n_above = above;
    return 0;
}
