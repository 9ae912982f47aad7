/* Assembly of (alpha I + K) on the structured grid (C, host, FP64).
 *
 * Isotropic (homogeneous_sigma_assembly_matrix, matrix_assembly.c:334-387):
 * every face between two active cells couples them with
 *     c = sigma_h * (area / distance),
 *     sigma_h = 2 s1 s2 / (s1 + s2)   (0 when either is 0)
 * (assembly_common.c:41-78,969-991); the row's diagonal is alpha + sum c.
 *
 * Anisotropic (anisotropic_sigma_assembly_matrix, matrix_assembly.c:389-514):
 * each cell carries D = sigma_l f f^T + sigma_t s s^T + sigma_n n n^T and its
 * row is built by mb_aniso_row, a restatement of fill_elements_aniso
 * (assembly_common.c:437-889) including its face averages of the
 * off-diagonal conductivities.  With the fibre in the xy plane and no removed
 * cells, a row depends only on the cell's z-plane and on which of the x/y
 * domain faces it touches, so the operator is stored as nz x 9 rows of 27
 * coefficients (the class table read by the stencil kernels).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "mb_internal.h"
#include "mb_assembly.h"

/* Harmonic mean of two face conductivities (assembly_common.c:971-991). */
static double harmonic(double s1, double s2) {
    if (s1 != 0.0 && s2 != 0.0) return (2.0f * s1 * s2) / (s1 + s2);
    return 0.0;
}

void mb_fibre_tensor(const double f[3], const double s[3], const double n[3], double sigma_l, double sigma_t,
                     double sigma_n, double D[3][3]) {
    if (sigma_t == sigma_n || !s || !n) {
        /* calc_tensor2 (assembly_common.c:1125-1139) */
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) D[i][j] = (sigma_l - sigma_t) * (f[i] * f[j]) + (i == j ? sigma_t : 0.0);
    } else {
        /* calc_tensor (assembly_common.c:1102-1123) */
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                D[i][j] = (sigma_l * (f[i] * f[j]) + sigma_t * (s[i] * s[j])) + sigma_n * (n[i] * n[j]);
    }
}

/* ---- restatement of fill_elements_aniso ------------------------------------ */

/* Offsets of the reference's 26 directions, in its enum order
 * (alg/cell/cell.h:22-50): RIGHT = +x, TOP = +y, FRONT = +z. */
enum { D_FRONT, D_BACK, D_TOP, D_DOWN, D_RIGHT, D_LEFT, D_FRONT_TOP, D_FRONT_DOWN, D_FRONT_RIGHT, D_FRONT_LEFT,
       D_FRONT_TOP_RIGHT, D_FRONT_TOP_LEFT, D_FRONT_DOWN_RIGHT, D_FRONT_DOWN_LEFT, D_BACK_TOP, D_BACK_DOWN,
       D_BACK_RIGHT, D_BACK_LEFT, D_BACK_TOP_RIGHT, D_BACK_TOP_LEFT, D_BACK_DOWN_RIGHT, D_BACK_DOWN_LEFT,
       D_TOP_RIGHT, D_TOP_LEFT, D_DOWN_RIGHT, D_DOWN_LEFT, D_NUM };

static const int dir_off[D_NUM][3] = {
    {0, 0, 1},   {0, 0, -1},  {0, 1, 0},   {0, -1, 0},  {1, 0, 0},   {-1, 0, 0},  {0, 1, 1},
    {0, -1, 1},  {1, 0, 1},   {-1, 0, 1},  {1, 1, 1},   {-1, 1, 1},  {1, -1, 1},  {-1, -1, 1},
    {0, 1, -1},  {0, -1, -1}, {1, 0, -1},  {-1, 0, -1}, {1, 1, -1},  {-1, 1, -1}, {1, -1, -1},
    {-1, -1, -1}, {1, 1, 0},  {-1, 1, 0},  {1, -1, 0},  {-1, -1, 0}};

static int slot(int d) { return (dir_off[d][2] + 1) * 9 + (dir_off[d][1] + 1) * 3 + (dir_off[d][0] + 1); }

enum { C_XY, C_XZ, C_YZ };

static double comp(const mb_nb_sigma *c, int which) {
    return which == C_XY ? c->xy : (which == C_XZ ? c->xz : c->yz);
}

/* Average of an off-diagonal component over the neighbour pairs that both
 * exist; returns the sum divided by the count, and the count. */
static double partial_sigma(const mb_nb_sigma nb[27], const int pairs[12], int which, int *count) {
    double s = 0.0;
    int c = 0;
    for (int q = 0; q < 12; q += 2) {
        const mb_nb_sigma *a = &nb[slot(pairs[q])], *b = &nb[slot(pairs[q + 1])];
        if (a->exists && b->exists) {
            s += comp(a, which) + comp(b, which);
            c += 2;
        }
    }
    if (c) s /= c;
    *count = c;
    return s;
}

/* sigma averaged over the two cells of a face plus the two partial averages
 * of the cross terms (calc_sigmas, assembly_common.c:115-405). */
typedef struct face_sig { double s1, s2, s3; int c1, c2, c3; } face_sig;

static face_sig face_sigmas(const mb_nb_sigma nb[27], int dir) {
    static const int P[6][2][12] = {
        /* FRONT: xz, yz */
        {{D_RIGHT, D_LEFT, D_FRONT_RIGHT, D_FRONT_LEFT, D_TOP_RIGHT, D_TOP_LEFT, D_FRONT_TOP_RIGHT, D_FRONT_TOP_LEFT,
          D_DOWN_RIGHT, D_DOWN_LEFT, D_FRONT_DOWN_RIGHT, D_FRONT_DOWN_LEFT},
         {D_TOP, D_DOWN, D_FRONT_TOP, D_FRONT_DOWN, D_TOP_RIGHT, D_DOWN_RIGHT, D_FRONT_TOP_RIGHT, D_FRONT_DOWN_RIGHT,
          D_TOP_LEFT, D_DOWN_LEFT, D_FRONT_TOP_LEFT, D_FRONT_DOWN_LEFT}},
        /* BACK: xz, yz */
        {{D_RIGHT, D_LEFT, D_BACK_RIGHT, D_BACK_LEFT, D_TOP_RIGHT, D_TOP_LEFT, D_BACK_TOP_RIGHT, D_BACK_TOP_LEFT,
          D_DOWN_RIGHT, D_DOWN_LEFT, D_BACK_DOWN_RIGHT, D_BACK_DOWN_LEFT},
         {D_TOP, D_DOWN, D_BACK_TOP, D_BACK_DOWN, D_TOP_RIGHT, D_DOWN_RIGHT, D_BACK_TOP_RIGHT, D_BACK_DOWN_RIGHT,
          D_TOP_LEFT, D_DOWN_LEFT, D_BACK_TOP_LEFT, D_BACK_DOWN_LEFT}},
        /* TOP: xy, yz */
        {{D_RIGHT, D_LEFT, D_TOP_RIGHT, D_TOP_LEFT, D_FRONT_RIGHT, D_FRONT_LEFT, D_FRONT_TOP_RIGHT, D_FRONT_TOP_LEFT,
          D_BACK_RIGHT, D_BACK_LEFT, D_BACK_TOP_RIGHT, D_BACK_TOP_LEFT},
         {D_FRONT, D_BACK, D_FRONT_TOP, D_BACK_TOP, D_FRONT_RIGHT, D_BACK_RIGHT, D_FRONT_TOP_RIGHT, D_BACK_TOP_RIGHT,
          D_FRONT_LEFT, D_BACK_LEFT, D_FRONT_TOP_LEFT, D_BACK_TOP_LEFT}},
        /* DOWN: xy, yz */
        {{D_RIGHT, D_LEFT, D_DOWN_RIGHT, D_DOWN_LEFT, D_FRONT_RIGHT, D_FRONT_LEFT, D_FRONT_DOWN_RIGHT,
          D_FRONT_DOWN_LEFT, D_BACK_RIGHT, D_BACK_LEFT, D_BACK_DOWN_RIGHT, D_BACK_DOWN_LEFT},
         {D_FRONT, D_BACK, D_FRONT_DOWN, D_BACK_DOWN, D_FRONT_RIGHT, D_BACK_RIGHT, D_FRONT_DOWN_RIGHT,
          D_BACK_DOWN_RIGHT, D_FRONT_LEFT, D_BACK_LEFT, D_FRONT_DOWN_LEFT, D_BACK_DOWN_LEFT}},
        /* RIGHT: xy, xz */
        {{D_TOP, D_DOWN, D_TOP_RIGHT, D_DOWN_RIGHT, D_FRONT_TOP, D_FRONT_DOWN, D_FRONT_TOP_RIGHT, D_FRONT_DOWN_RIGHT,
          D_BACK_TOP, D_BACK_DOWN, D_BACK_TOP_RIGHT, D_BACK_DOWN_RIGHT},
         {D_FRONT, D_BACK, D_FRONT_RIGHT, D_BACK_RIGHT, D_FRONT_TOP, D_BACK_TOP, D_FRONT_TOP_RIGHT, D_BACK_TOP_RIGHT,
          D_FRONT_DOWN, D_BACK_DOWN, D_FRONT_DOWN_RIGHT, D_BACK_DOWN_RIGHT}},
        /* LEFT: xy, xz */
        {{D_TOP, D_DOWN, D_TOP_LEFT, D_DOWN_LEFT, D_FRONT_TOP, D_FRONT_DOWN, D_FRONT_TOP_LEFT, D_FRONT_DOWN_LEFT,
          D_BACK_TOP, D_BACK_DOWN, D_BACK_TOP_LEFT, D_BACK_DOWN_LEFT},
         {D_FRONT, D_BACK, D_FRONT_LEFT, D_BACK_LEFT, D_FRONT_TOP, D_BACK_TOP, D_FRONT_TOP_LEFT, D_BACK_TOP_LEFT,
          D_FRONT_DOWN, D_BACK_DOWN, D_FRONT_DOWN_LEFT, D_BACK_DOWN_LEFT}},
    };
    /* which cross components the two partial averages use */
    static const int W[6][2] = {{C_XZ, C_YZ}, {C_XZ, C_YZ}, {C_XY, C_YZ}, {C_XY, C_YZ}, {C_XY, C_XZ}, {C_XY, C_XZ}};
    face_sig f = {0, 0, 0, 0, 0, 0};
    const mb_nb_sigma *c = &nb[13], *o = &nb[slot(dir)];
    if (!o->exists) return f;
    double a, b;
    if (dir == D_RIGHT || dir == D_LEFT) { a = o->x; b = c->x; }
    else if (dir == D_TOP || dir == D_DOWN) { a = o->y; b = c->y; }
    else { a = o->z; b = c->z; }
    f.s1 = (a + b) / 2.0;
    f.c1 = 1;
    f.s2 = partial_sigma(nb, P[dir][0], W[dir][0], &f.c2);
    f.s3 = partial_sigma(nb, P[dir][1], W[dir][1], &f.c3);
    return f;
}

/* DIVIDE (assembly_common.c:407-412): the partial averages are divided by
 * their count a second time where they enter the coefficients. */
static double DV(double num, int den) { return den != 0 ? num / den : 0.0; }

void mb_aniso_row(const mb_nb_sigma nb[27], double dx, double dy, double dz, double alpha, double row[27]) {
    for (int q = 0; q < 27; ++q) row[q] = 0.0;
    const double yzx = (dy * dz) / dx, xzy = (dx * dz) / dy, xyz = (dx * dy) / dz;
    const face_sig R = face_sigmas(nb, D_RIGHT), L = face_sigmas(nb, D_LEFT);
    const face_sig T = face_sigmas(nb, D_TOP), Dn = face_sigmas(nb, D_DOWN);
    const face_sig F = face_sigmas(nb, D_FRONT), B = face_sigmas(nb, D_BACK);
    /* names follow the reference: sigma_<comp>_j<axis>_<face> */
    const double xy_jx_r = DV(R.s2, R.c2), xz_jx_r = DV(R.s3, R.c3);
    const double xy_jx_l = DV(L.s2, L.c2), xz_jx_l = DV(L.s3, L.c3);
    const double xy_jy_t = DV(T.s2, T.c2), yz_jy_t = DV(T.s3, T.c3);
    const double xy_jy_d = DV(Dn.s2, Dn.c2), yz_jy_d = DV(Dn.s3, Dn.c3);
    const double xz_jz_f = DV(F.s2, F.c2), yz_jz_f = DV(F.s3, F.c3);
    const double xz_jz_b = DV(B.s2, B.c2), yz_jz_b = DV(B.s3, B.c3);

    row[13] = alpha + (yzx * R.s1 + yzx * L.s1 + xzy * T.s1 + xzy * Dn.s1 + xyz * F.s1 + xyz * B.s1);

#define EX(d) (nb[slot(d)].exists)
#define ADD(d, v) do { const double v_ = (v); if (v_ != 0) row[slot(d)] += v_; } while (0)
    for (int d = 0; d < D_NUM; ++d) {
        if (!EX(d)) continue;
        double v = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        switch (d) {
        case D_FRONT:
            v += -F.s1 * xyz;
            if (EX(D_BACK)) v += -yz_jy_t * dx + yz_jy_d * dx - xz_jx_r * dy + xz_jx_l * dy;
            break;
        case D_BACK:
            v += -B.s1 * xyz;
            if (EX(D_FRONT)) v += yz_jy_t * dx - yz_jy_d * dx + xz_jx_r * dy - xz_jx_l * dy;
            break;
        case D_TOP:
            v += -T.s1 * xzy;
            if (EX(D_DOWN)) v += -yz_jz_f * dx + yz_jz_b * dx - xy_jx_r * dz + xy_jx_l * dz;
            break;
        case D_DOWN:
            v += -Dn.s1 * xzy;
            if (EX(D_TOP)) v += yz_jz_f * dx - yz_jz_b * dx + xy_jx_r * dz - xy_jx_l * dz;
            break;
        case D_RIGHT:
            v += -R.s1 * yzx;
            if (EX(D_LEFT)) v += -xz_jz_f * dy + xz_jz_b * dy - xy_jy_t * dz + xy_jy_d * dz;
            break;
        case D_LEFT:
            v += -L.s1 * yzx;
            if (EX(D_RIGHT)) v += xz_jz_f * dy - xz_jz_b * dy + xy_jy_t * dz - xy_jy_d * dz;
            break;
        case D_FRONT_TOP:
            if (EX(D_FRONT_DOWN)) { s1 += -xy_jx_r * dz + xy_jx_l * dz - yz_jz_f * dx; ADD(D_FRONT_DOWN, -s1); }
            if (EX(D_BACK_TOP)) { s2 += -yz_jy_t * dx - xz_jx_r * dy + xz_jx_l * dy; ADD(D_BACK_TOP, -s2); }
            v += s1 + s2;
            break;
        case D_FRONT_DOWN:
            if (EX(D_BACK_DOWN)) {
                s1 += yz_jy_d * dx - xz_jx_r * dy + xz_jx_l * dy;
                ADD(D_FRONT_DOWN, s1); ADD(D_BACK_DOWN, -s1);
            }
            break;
        case D_BACK_TOP:
            if (EX(D_BACK_DOWN)) {
                s1 += yz_jz_b * dx - xy_jx_r * dz + xy_jx_l * dz;
                ADD(D_BACK_TOP, s1); ADD(D_BACK_DOWN, -s1);
            }
            break;
        case D_FRONT_RIGHT:
            if (EX(D_BACK_RIGHT)) { s1 += -xz_jx_r * dy - yz_jy_t * dx + yz_jy_d * dx; ADD(D_BACK_RIGHT, -s1); }
            if (EX(D_FRONT_LEFT)) { s2 += -xz_jz_f * dy - xy_jy_t * dz + xy_jy_d * dz; ADD(D_FRONT_LEFT, -s2); }
            v += s1 + s2;
            break;
        case D_FRONT_LEFT:
            if (EX(D_BACK_LEFT)) {
                s1 += -yz_jy_t * dx + yz_jy_d * dx + xz_jx_l * dy;
                ADD(D_FRONT_LEFT, s1); ADD(D_BACK_LEFT, -s1);
            }
            break;
        case D_BACK_RIGHT:
            if (EX(D_BACK_LEFT)) {
                s1 += xz_jz_b * dy - xy_jy_t * dz + xy_jy_d * dz;
                ADD(D_BACK_RIGHT, s1); ADD(D_BACK_LEFT, -s1);
            }
            break;
        case D_TOP_RIGHT:
            if (EX(D_DOWN_RIGHT)) { s1 += -xy_jx_r * dz - yz_jz_f * dx + yz_jz_b * dx; ADD(D_DOWN_RIGHT, -s1); }
            if (EX(D_TOP_LEFT)) { s2 += -xz_jz_f * dy + xz_jz_b * dy - xy_jy_t * dz; ADD(D_TOP_LEFT, -s2); }
            v += s1 + s2;
            break;
        case D_TOP_LEFT:
            if (EX(D_DOWN_LEFT)) {
                s1 += -yz_jz_f * dx + yz_jz_b * dx + xy_jx_l * dz;
                ADD(D_TOP_LEFT, s1); ADD(D_DOWN_LEFT, -s1);
            }
            break;
        case D_DOWN_RIGHT:
            if (EX(D_DOWN_LEFT)) {
                s1 += -xz_jz_f * dy + xz_jz_b * dy + xy_jy_d * dz;
                ADD(D_DOWN_RIGHT, s1); ADD(D_DOWN_LEFT, -s1);
            }
            break;
        case D_FRONT_TOP_RIGHT:
            if (EX(D_FRONT_DOWN_RIGHT)) { s1 += -xy_jx_r * dz - yz_jz_f * dx; ADD(D_FRONT_DOWN_RIGHT, -s1); }
            if (EX(D_BACK_TOP_RIGHT)) { s2 += -xz_jx_r * dy - yz_jy_t * dx; ADD(D_BACK_TOP_RIGHT, -s2); }
            if (EX(D_FRONT_TOP_LEFT)) { s3 += -xz_jz_f * dy - xy_jy_t * dz; ADD(D_FRONT_TOP_LEFT, -s3); }
            v += s1 + s2 + s3;
            break;
        case D_FRONT_TOP_LEFT:
            if (EX(D_FRONT_DOWN_LEFT)) {
                s1 += xy_jx_l * dz - yz_jz_f * dx;
                ADD(D_FRONT_TOP_LEFT, s1); ADD(D_FRONT_DOWN_LEFT, -s1);
            }
            if (EX(D_BACK_TOP_LEFT)) {
                s2 += xz_jx_l * dy - yz_jy_t * dx;
                ADD(D_FRONT_TOP_LEFT, s2); ADD(D_BACK_TOP_LEFT, -s2);
            }
            break;
        case D_FRONT_DOWN_RIGHT:
            if (EX(D_BACK_DOWN_RIGHT)) {
                s1 += -xz_jx_r * dy + yz_jy_d * dx;
                ADD(D_FRONT_DOWN_RIGHT, s1); ADD(D_BACK_DOWN_RIGHT, -s1);
            }
            if (EX(D_FRONT_DOWN_LEFT)) {
                s2 += xy_jy_d * dz - xz_jz_f * dy;
                ADD(D_FRONT_DOWN_RIGHT, s2); ADD(D_FRONT_DOWN_LEFT, -s2);
            }
            break;
        case D_FRONT_DOWN_LEFT:
            if (EX(D_BACK_DOWN_LEFT)) {
                s1 += xz_jx_l * dy + yz_jy_d * dx;
                ADD(D_FRONT_DOWN_LEFT, s1); ADD(D_BACK_DOWN_LEFT, -s1);
            }
            break;
        case D_BACK_TOP_RIGHT:
            if (EX(D_BACK_DOWN_RIGHT)) {
                s1 += -xy_jx_r * dz + yz_jz_b * dx;
                ADD(D_BACK_TOP_RIGHT, s1); ADD(D_BACK_DOWN_RIGHT, -s1);
            }
            if (EX(D_BACK_TOP_LEFT)) {
                s2 += -xy_jy_t * dz + xz_jz_b * dy;
                ADD(D_BACK_TOP_RIGHT, s2); ADD(D_BACK_TOP_LEFT, -s2);
            }
            break;
        case D_BACK_TOP_LEFT:
            if (EX(D_BACK_DOWN_LEFT)) {
                s1 += xy_jx_l * dz + yz_jz_b * dx;
                ADD(D_BACK_TOP_LEFT, s1); ADD(D_BACK_DOWN_LEFT, -s1);
            }
            break;
        case D_BACK_DOWN_RIGHT:
            if (EX(D_BACK_DOWN_LEFT)) {
                s1 += xy_jy_d * dz + xz_jz_b * dy;
                ADD(D_BACK_DOWN_RIGHT, s1); ADD(D_BACK_DOWN_LEFT, -s1);
            }
            break;
        default:
            break;
        }
        if (v != 0.0) row[slot(d)] += v;
    }
#undef EX
#undef ADD
}

/* ---- operator assembly for a descriptor --------------------------------- */

static void plane_tensor(const mb_monodomain_desc *d, int k, mb_nb_sigma *t) {
    const double th = d->fibre_angle_z ? d->fibre_angle_z[k] : 0.0;
    const double f[3] = {cos(th), sin(th), 0.0};
    const double s[3] = {-sin(th), cos(th), 0.0};
    const double n[3] = {0.0, 0.0, 1.0};
    double D[3][3];
    mb_fibre_tensor(f, s, n, d->sigma_l, d->sigma_t, d->sigma_n, D);
    t->exists = 1;
    t->x = D[0][0]; t->y = D[1][1]; t->z = D[2][2];
    t->xy = D[0][1]; t->xz = D[0][2]; t->yz = D[1][2];
}

int mb_assemble(const mb_monodomain_desc *d, mb_assembly_out *out) {
    memset(out, 0, sizeof *out);
    const int64_t n = (int64_t)d->nx * d->ny * d->nz;
    if (d->assembly == MB_ASSEMBLY_HOMOGENEOUS) {
        out->kind = 0;
        out->cx = harmonic(d->sigma[0], d->sigma[0]) * ((d->dy * d->dz) / d->dx);
        out->cy = harmonic(d->sigma[1], d->sigma[1]) * ((d->dx * d->dz) / d->dy);
        out->cz = harmonic(d->sigma[2], d->sigma[2]) * ((d->dx * d->dy) / d->dz);
        return MB_OK;
    }
    if (d->assembly == MB_ASSEMBLY_PER_CELL_SIGMA) {
        if (!d->sigma_cell) return MB_ERR_ARG;
        out->kind = 1;
        out->fx = (double *)calloc((size_t)n, sizeof(double));
        out->fy = (double *)calloc((size_t)n, sizeof(double));
        out->fz = (double *)calloc((size_t)n, sizeof(double));
        if (!out->fx || !out->fy || !out->fz) return MB_ERR_NOMEM;
        const double mx = (d->dy * d->dz) / d->dx, my = (d->dx * d->dz) / d->dy, mz = (d->dx * d->dy) / d->dz;
        const int64_t sy = d->nx, sz = (int64_t)d->nx * d->ny;
        for (int k = 0; k < d->nz; ++k)
            for (int j = 0; j < d->ny; ++j)
                for (int i = 0; i < d->nx; ++i) {
                    const int64_t g = i + sy * j + sz * k;
                    const int a = !d->active || d->active[g];
                    if (!a) continue;
                    if (i + 1 < d->nx && (!d->active || d->active[g + 1]))
                        out->fx[g] = harmonic(d->sigma_cell[g], d->sigma_cell[g + 1]) * mx;
                    if (j + 1 < d->ny && (!d->active || d->active[g + sy]))
                        out->fy[g] = harmonic(d->sigma_cell[g], d->sigma_cell[g + sy]) * my;
                    if (k + 1 < d->nz && (!d->active || d->active[g + sz]))
                        out->fz[g] = harmonic(d->sigma_cell[g], d->sigma_cell[g + sz]) * mz;
                }
        return MB_OK;
    }
    if (d->assembly != MB_ASSEMBLY_ANISOTROPIC) return MB_ERR_ARG;
    if (d->nx < 1 || d->ny < 1 || d->nz < 1) return MB_ERR_ARG;

    /* per-plane tensors; cross terms present? */
    int cross = 0;
    mb_nb_sigma *pt = (mb_nb_sigma *)malloc((size_t)d->nz * sizeof(mb_nb_sigma));
    if (!pt) return MB_ERR_NOMEM;
    for (int k = 0; k < d->nz; ++k) {
        plane_tensor(d, k, &pt[k]);
        if (pt[k].xy != 0.0 || pt[k].xz != 0.0 || pt[k].yz != 0.0) cross = 1;
        if (pt[k].x != pt[0].x || pt[k].y != pt[0].y || pt[k].z != pt[0].z) cross = 1;
    }
    if (!cross) {
        /* diagonal, uniform tensor: the face average (s + s)/2 = s, no cross
         * terms; the operator is the constant 7-point one */
        out->kind = 0;
        out->cx = ((pt[0].x + pt[0].x) / 2.0) * ((d->dy * d->dz) / d->dx);
        out->cy = ((pt[0].y + pt[0].y) / 2.0) * ((d->dx * d->dz) / d->dy);
        out->cz = ((pt[0].z + pt[0].z) / 2.0) * ((d->dx * d->dy) / d->dz);
        free(pt);
        return MB_OK;
    }
    if (d->active) {
        free(pt);
        return MB_ERR_UNSUPPORTED;   /* per-plane rows assume every cell active */
    }
    out->kind = 2;
    out->table = (double *)calloc((size_t)d->nz * 9 * 27, sizeof(double));
    if (!out->table) { free(pt); return MB_ERR_NOMEM; }
    const double alpha = mb_alpha(d->beta, d->cm, d->dt_pde, d->dx, d->dy, d->dz);
    for (int k = 0; k < d->nz; ++k)
        for (int cy = 0; cy < 3; ++cy)
            for (int cx = 0; cx < 3; ++cx) {
                mb_nb_sigma nb[27];
                for (int oz = -1; oz <= 1; ++oz)
                    for (int oy = -1; oy <= 1; ++oy)
                        for (int ox = -1; ox <= 1; ++ox) {
                            const int q = (oz + 1) * 9 + (oy + 1) * 3 + (ox + 1);
                            int ex = 1;
                            if (k + oz < 0 || k + oz >= d->nz) ex = 0;
                            if (ox == -1 && (cx == 0)) ex = 0;
                            if (ox == 1 && (cx == 2 || (cx == 0 && d->nx < 2))) ex = 0;
                            if (oy == -1 && (cy == 0)) ex = 0;
                            if (oy == 1 && (cy == 2 || (cy == 0 && d->ny < 2))) ex = 0;
                            if (ex) nb[q] = pt[k + oz];
                            else memset(&nb[q], 0, sizeof nb[q]);
                        }
                mb_aniso_row(nb, d->dx, d->dy, d->dz, alpha, out->table + ((size_t)k * 9 + cy * 3 + cx) * 27);
            }
    free(pt);
    return MB_OK;
}

void mb_assembly_free(mb_assembly_out *out) {
    free(out->fx); free(out->fy); free(out->fz); free(out->table);
    memset(out, 0, sizeof *out);
}
