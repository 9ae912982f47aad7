/* Assembly of (alpha I + K) as a CSR matrix, FP64 -- TEST INFRASTRUCTURE
 * (oracle).  Restates src/matrix_assembly_library/matrix_assembly.c and
 * assembly_common.c for a structured cuboid whose cells all have the same
 * size (one refinement level, so every neighbour is found directly):
 *
 *   initialize_diagonal_elements (assembly_common.c:4-39): row diagonal = alpha
 *   homogeneous_sigma_assembly_matrix (matrix_assembly.c:334-387) with
 *     fill_discretization_matrix_elements / fill_element
 *     (assembly_common.c:41-78,911-1048): every face between two active cells
 *     couples them with sigma_h * area / distance, sigma_h the harmonic mean
 *     2.0f s1 s2 / (s1 + s2) of the two cells' sigma on that axis (0 if either
 *     is 0)
 *   anisotropic_sigma_assembly_matrix (matrix_assembly.c:389-514) with
 *     calc_tensor / calc_tensor2 (assembly_common.c:1102-1139), calc_sigmas
 *     (:115-411), DIVIDE (:414-419), fill_elements_aniso (:437-830) and
 *     fill_discretization_matrix_elements_aniso (:892-908)
 *
 * Rows are the active cells in grid order; the diagonal is each row's first
 * entry; entries that are exactly 0 are dropped (as the reference never
 * stores them).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* ALPHA (monodomain/constants.h:11) with UM2_TO_CM2 = 1e-8 written as a float
 * literal in the reference. */
static double alpha_of(const mb_monodomain_desc *d) {
    return (((d->beta * d->cm) / d->dt_pde) * (double)1.0e-8f) * (d->dx * d->dy * d->dz);
}

typedef struct grid_view {
    int nx, ny, nz;
    const uint8_t *active;
} grid_view;

static int cell_at(const grid_view *G, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= G->nx || j >= G->ny || k >= G->nz) return -1;
    const int g = i + G->nx * (j + G->ny * k);
    if (G->active && !G->active[g]) return -1;
    return g;
}

/* A row under construction: at most 27 distinct columns (duplicates of a
 * column, which the reference may append, are summed: the product A x is
 * the same). */
typedef struct row27 {
    int n;
    int32_t col[27];
    double val[27];
} row27;

static void row_add(row27 *r, int32_t col, double v) {
    for (int q = 0; q < r->n; ++q)
        if (r->col[q] == col) {
            r->val[q] += v;
            return;
        }
    r->col[r->n] = col;
    r->val[r->n] = v;
    r->n++;
}

/* ---- homogeneous / per-cell isotropic sigma --------------------------------- */

static double harmonic(double s1, double s2) {
    if (s1 != 0.0 && s2 != 0.0) return (2.0f * s1 * s2) / (s1 + s2);
    return 0.0;
}

static void homogeneous_row(const mb_monodomain_desc *d, const grid_view *G, int i, int j, int k, double alpha,
                            row27 *r) {
    const int g = i + G->nx * (j + G->ny * k);
    r->n = 0;
    row_add(r, g, alpha);
    /* the reference visits BACK, FRONT, TOP, DOWN, RIGHT, LEFT
     * (matrix_assembly.c:362-381) */
    static const int off[6][3] = {{0, 0, -1}, {0, 0, 1}, {0, 1, 0}, {0, -1, 0}, {1, 0, 0}, {-1, 0, 0}};
    for (int q = 0; q < 6; ++q) {
        const int gn = cell_at(G, i + off[q][0], j + off[q][1], k + off[q][2]);
        if (gn < 0) continue;
        double s_c, s_n, mult;
        const int axis = off[q][0] ? 0 : (off[q][1] ? 1 : 2);
        if (d->assembly == MB_ASSEMBLY_PER_CELL_SIGMA) {
            s_c = d->sigma_cell[g];
            s_n = d->sigma_cell[gn];
        } else {
            s_c = s_n = d->sigma[axis];
        }
        if (axis == 0) mult = (d->dy * d->dz) / d->dx;
        else if (axis == 1) mult = (d->dx * d->dz) / d->dy;
        else mult = (d->dx * d->dy) / d->dz;
        const double s = harmonic(s_c, s_n);
        row_add(r, gn, -s * mult);
        r->val[0] += s * mult;
    }
}

/* ---- anisotropic ---------------------------------------------------------------- */

typedef struct tensor6 { double x, y, z, xy, xz, yz; } tensor6;

/* calc_tensor2 when sigma_t == sigma_n, else calc_tensor, with the fibre in
 * the xy plane at angle theta: f = (cos, sin, 0), s = (-sin, cos, 0),
 * n = (0, 0, 1). */
static tensor6 fibre_tensor(double theta, double sl, double st, double sn) {
    const double f[3] = {cos(theta), sin(theta), 0.0};
    const double s[3] = {-sin(theta), cos(theta), 0.0};
    const double n[3] = {0.0, 0.0, 1.0};
    double D[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            if (st == sn) D[a][b] = (sl - st) * (f[a] * f[b]) + (a == b ? st : 0.0);
            else D[a][b] = (sl * (f[a] * f[b]) + st * (s[a] * s[b])) + sn * (n[a] * n[b]);
        }
    tensor6 t = {D[0][0], D[1][1], D[2][2], D[0][1], D[0][2], D[1][2]};
    return t;
}

static double comp_of(const tensor6 *t, int which) { return which == 0 ? t->xy : (which == 1 ? t->xz : t->yz); }

/* The cell's 3x3x3 neighbourhood: ex[dz+1][dy+1][dx+1] = active neighbour. */
typedef struct hood {
    int g[3][3][3];
    const tensor6 *t[3][3][3];
} hood;

#define H_EX(h, ox, oy, oz) ((h)->g[(oz) + 1][(oy) + 1][(ox) + 1] >= 0)

/* CALC_PARTIAL_SIGMA (assembly_common.c:78-113) over the six pairs the
 * reference lists for a face (calc_sigmas, :115-411): with face offset D along
 * axis a, cross axis b and third axis c, the pairs are (B + e_b, B - e_b) for
 * B in {0, D, +e_c, D + e_c, -e_c, D - e_c}; a pair counts when both of its
 * cells are active neighbours. */
static void partial_sigma(const hood *h, const int D[3], int b, int c, int which, double *sum, int *count) {
    const int bases[6][3] = {{0, 0, 0}, {D[0], D[1], D[2]}, {0, 0, 0}, {D[0], D[1], D[2]}, {0, 0, 0},
                             {D[0], D[1], D[2]}};
    double s = 0.0;
    int n = 0;
    for (int q = 0; q < 6; ++q) {
        int B[3] = {bases[q][0], bases[q][1], bases[q][2]};
        if (q == 2 || q == 3) B[c] += 1;
        if (q == 4 || q == 5) B[c] -= 1;
        int P[3] = {B[0], B[1], B[2]}, M[3] = {B[0], B[1], B[2]};
        P[b] += 1;
        M[b] -= 1;
        if (H_EX(h, P[0], P[1], P[2]) && H_EX(h, M[0], M[1], M[2])) {
            s += comp_of(h->t[P[2] + 1][P[1] + 1][P[0] + 1], which) + comp_of(h->t[M[2] + 1][M[1] + 1][M[0] + 1], which);
            n += 2;
        }
    }
    if (n) s /= n;
    *sum = s;
    *count = n;
}

/* calc_sigmas for one face: s1 = arithmetic mean of the diagonal component,
 * s2 / s3 = the two partial cross averages and their counts. */
typedef struct face { double s1, s2, s3; int n2, n3; } face;

static face face_sigmas(const hood *h, int ox, int oy, int oz) {
    face f = {0.0, 0.0, 0.0, 0, 0};
    if (!H_EX(h, ox, oy, oz)) return f;
    const tensor6 *tc = h->t[1][1][1], *tn = h->t[oz + 1][oy + 1][ox + 1];
    const int D[3] = {ox, oy, oz};
    if (ox) {        /* RIGHT / LEFT: xy (b = y, c = z), xz (b = z, c = y) */
        f.s1 = (tn->x + tc->x) / 2.0;
        partial_sigma(h, D, 1, 2, 0, &f.s2, &f.n2);
        partial_sigma(h, D, 2, 1, 1, &f.s3, &f.n3);
    } else if (oy) { /* TOP / DOWN: xy (b = x, c = z), yz (b = z, c = x) */
        f.s1 = (tn->y + tc->y) / 2.0;
        partial_sigma(h, D, 0, 2, 0, &f.s2, &f.n2);
        partial_sigma(h, D, 2, 0, 2, &f.s3, &f.n3);
    } else {         /* FRONT / BACK: xz (b = x, c = y), yz (b = y, c = x) */
        f.s1 = (tn->z + tc->z) / 2.0;
        partial_sigma(h, D, 0, 1, 1, &f.s2, &f.n2);
        partial_sigma(h, D, 1, 0, 2, &f.s3, &f.n3);
    }
    return f;
}

static double DIVIDE(double num, int den) { return den != 0 ? num / den : 0.0; }

/* fill_elements_aniso (assembly_common.c:437-830) for the cell at (i,j,k).
 * Directions are offsets: +x RIGHT, +y TOP, +z FRONT (alg/cell/cell.h). */
static void aniso_row(const mb_monodomain_desc *d, const grid_view *G, const tensor6 *tens, int i, int j, int k,
                      double alpha, row27 *r) {
    hood h;
    for (int c = -1; c <= 1; ++c)
        for (int b = -1; b <= 1; ++b)
            for (int a = -1; a <= 1; ++a) {
                const int gn = (a || b || c) ? cell_at(G, i + a, j + b, k + c) : i + G->nx * (j + G->ny * k);
                h.g[c + 1][b + 1][a + 1] = gn;
                h.t[c + 1][b + 1][a + 1] = gn >= 0 ? &tens[gn] : NULL;
            }
    const double dx = d->dx, dy = d->dy, dz = d->dz;
    const double yzx = (dy * dz) / dx, xzy = (dx * dz) / dy, xyz = (dx * dy) / dz;
    const face R = face_sigmas(&h, 1, 0, 0), L = face_sigmas(&h, -1, 0, 0);
    const face T = face_sigmas(&h, 0, 1, 0), Dn = face_sigmas(&h, 0, -1, 0);
    const face F = face_sigmas(&h, 0, 0, 1), B = face_sigmas(&h, 0, 0, -1);
    const double xy_jx_r = DIVIDE(R.s2, R.n2), xz_jx_r = DIVIDE(R.s3, R.n3);
    const double xy_jx_l = DIVIDE(L.s2, L.n2), xz_jx_l = DIVIDE(L.s3, L.n3);
    const double xy_jy_t = DIVIDE(T.s2, T.n2), yz_jy_t = DIVIDE(T.s3, T.n3);
    const double xy_jy_d = DIVIDE(Dn.s2, Dn.n2), yz_jy_d = DIVIDE(Dn.s3, Dn.n3);
    const double xz_jz_f = DIVIDE(F.s2, F.n2), yz_jz_f = DIVIDE(F.s3, F.n3);
    const double xz_jz_b = DIVIDE(B.s2, B.n2), yz_jz_b = DIVIDE(B.s3, B.n3);

    r->n = 0;
    row_add(r, h.g[1][1][1], alpha);
    r->val[0] += yzx * R.s1 + yzx * L.s1 + xzy * T.s1 + xzy * Dn.s1 + xyz * F.s1 + xyz * B.s1;

#define N(ox, oy, oz) H_EX(&h, ox, oy, oz)
#define ADD(ox, oy, oz, v)                                                      \
    do {                                                                       \
        const double v_ = (v);                                                 \
        if (v_ != 0) row_add(r, h.g[(oz) + 1][(oy) + 1][(ox) + 1], v_);        \
    } while (0)
    /* the faces */
    if (N(0, 0, 1)) { /* FRONT */
        double v = -F.s1 * xyz;
        if (N(0, 0, -1)) v += -yz_jy_t * dx + yz_jy_d * dx - xz_jx_r * dy + xz_jx_l * dy;
        ADD(0, 0, 1, v);
    }
    if (N(0, 0, -1)) { /* BACK */
        double v = -B.s1 * xyz;
        if (N(0, 0, 1)) v += yz_jy_t * dx - yz_jy_d * dx + xz_jx_r * dy - xz_jx_l * dy;
        ADD(0, 0, -1, v);
    }
    if (N(0, 1, 0)) { /* TOP */
        double v = -T.s1 * xzy;
        if (N(0, -1, 0)) v += -yz_jz_f * dx + yz_jz_b * dx - xy_jx_r * dz + xy_jx_l * dz;
        ADD(0, 1, 0, v);
    }
    if (N(0, -1, 0)) { /* DOWN */
        double v = -Dn.s1 * xzy;
        if (N(0, 1, 0)) v += yz_jz_f * dx - yz_jz_b * dx + xy_jx_r * dz - xy_jx_l * dz;
        ADD(0, -1, 0, v);
    }
    if (N(1, 0, 0)) { /* RIGHT */
        double v = -R.s1 * yzx;
        if (N(-1, 0, 0)) v += -xz_jz_f * dy + xz_jz_b * dy - xy_jy_t * dz + xy_jy_d * dz;
        ADD(1, 0, 0, v);
    }
    if (N(-1, 0, 0)) { /* LEFT */
        double v = -L.s1 * yzx;
        if (N(1, 0, 0)) v += xz_jz_f * dy - xz_jz_b * dy + xy_jy_t * dz - xy_jy_d * dz;
        ADD(-1, 0, 0, v);
    }
    /* the edges */
    if (N(0, 1, 1)) { /* FRONT_TOP */
        double s1 = 0.0, s2 = 0.0;
        if (N(0, -1, 1)) { s1 = -xy_jx_r * dz + xy_jx_l * dz - yz_jz_f * dx; ADD(0, -1, 1, -s1); }
        if (N(0, 1, -1)) { s2 = -yz_jy_t * dx - xz_jx_r * dy + xz_jx_l * dy; ADD(0, 1, -1, -s2); }
        ADD(0, 1, 1, s1 + s2);
    }
    if (N(0, -1, 1) && N(0, -1, -1)) { /* FRONT_DOWN */
        const double s1 = yz_jy_d * dx - xz_jx_r * dy + xz_jx_l * dy;
        ADD(0, -1, 1, s1); ADD(0, -1, -1, -s1);
    }
    if (N(0, 1, -1) && N(0, -1, -1)) { /* BACK_TOP */
        const double s1 = yz_jz_b * dx - xy_jx_r * dz + xy_jx_l * dz;
        ADD(0, 1, -1, s1); ADD(0, -1, -1, -s1);
    }
    if (N(1, 0, 1)) { /* FRONT_RIGHT */
        double s1 = 0.0, s2 = 0.0;
        if (N(1, 0, -1)) { s1 = -xz_jx_r * dy - yz_jy_t * dx + yz_jy_d * dx; ADD(1, 0, -1, -s1); }
        if (N(-1, 0, 1)) { s2 = -xz_jz_f * dy - xy_jy_t * dz + xy_jy_d * dz; ADD(-1, 0, 1, -s2); }
        ADD(1, 0, 1, s1 + s2);
    }
    if (N(-1, 0, 1) && N(-1, 0, -1)) { /* FRONT_LEFT */
        const double s1 = -yz_jy_t * dx + yz_jy_d * dx + xz_jx_l * dy;
        ADD(-1, 0, 1, s1); ADD(-1, 0, -1, -s1);
    }
    if (N(1, 0, -1) && N(-1, 0, -1)) { /* BACK_RIGHT */
        const double s1 = xz_jz_b * dy - xy_jy_t * dz + xy_jy_d * dz;
        ADD(1, 0, -1, s1); ADD(-1, 0, -1, -s1);
    }
    if (N(1, 1, 0)) { /* TOP_RIGHT */
        double s1 = 0.0, s2 = 0.0;
        if (N(1, -1, 0)) { s1 = -xy_jx_r * dz - yz_jz_f * dx + yz_jz_b * dx; ADD(1, -1, 0, -s1); }
        if (N(-1, 1, 0)) { s2 = -xz_jz_f * dy + xz_jz_b * dy - xy_jy_t * dz; ADD(-1, 1, 0, -s2); }
        ADD(1, 1, 0, s1 + s2);
    }
    if (N(-1, 1, 0) && N(-1, -1, 0)) { /* TOP_LEFT */
        const double s1 = -yz_jz_f * dx + yz_jz_b * dx + xy_jx_l * dz;
        ADD(-1, 1, 0, s1); ADD(-1, -1, 0, -s1);
    }
    if (N(1, -1, 0) && N(-1, -1, 0)) { /* DOWN_RIGHT */
        const double s1 = -xz_jz_f * dy + xz_jz_b * dy + xy_jy_d * dz;
        ADD(1, -1, 0, s1); ADD(-1, -1, 0, -s1);
    }
    /* the corners */
    if (N(1, 1, 1)) { /* FRONT_TOP_RIGHT */
        double s1 = 0.0, s2 = 0.0, s3 = 0.0;
        if (N(1, -1, 1)) { s1 = -xy_jx_r * dz - yz_jz_f * dx; ADD(1, -1, 1, -s1); }
        if (N(1, 1, -1)) { s2 = -xz_jx_r * dy - yz_jy_t * dx; ADD(1, 1, -1, -s2); }
        if (N(-1, 1, 1)) { s3 = -xz_jz_f * dy - xy_jy_t * dz; ADD(-1, 1, 1, -s3); }
        ADD(1, 1, 1, s1 + s2 + s3);
    }
    if (N(-1, 1, 1)) { /* FRONT_TOP_LEFT */
        if (N(-1, -1, 1)) {
            const double s1 = xy_jx_l * dz - yz_jz_f * dx;
            ADD(-1, 1, 1, s1); ADD(-1, -1, 1, -s1);
        }
        if (N(-1, 1, -1)) {
            const double s2 = xz_jx_l * dy - yz_jy_t * dx;
            ADD(-1, 1, 1, s2); ADD(-1, 1, -1, -s2);
        }
    }
    if (N(1, -1, 1)) { /* FRONT_DOWN_RIGHT */
        if (N(1, -1, -1)) {
            const double s1 = -xz_jx_r * dy + yz_jy_d * dx;
            ADD(1, -1, 1, s1); ADD(1, -1, -1, -s1);
        }
        if (N(-1, -1, 1)) {
            const double s2 = xy_jy_d * dz - xz_jz_f * dy;
            ADD(1, -1, 1, s2); ADD(-1, -1, 1, -s2);
        }
    }
    if (N(-1, -1, 1) && N(-1, -1, -1)) { /* FRONT_DOWN_LEFT */
        const double s1 = xz_jx_l * dy + yz_jy_d * dx;
        ADD(-1, -1, 1, s1); ADD(-1, -1, -1, -s1);
    }
    if (N(1, 1, -1)) { /* BACK_TOP_RIGHT */
        if (N(1, -1, -1)) {
            const double s1 = -xy_jx_r * dz + yz_jz_b * dx;
            ADD(1, 1, -1, s1); ADD(1, -1, -1, -s1);
        }
        if (N(-1, 1, -1)) {
            const double s2 = -xy_jy_t * dz + xz_jz_b * dy;
            ADD(1, 1, -1, s2); ADD(-1, 1, -1, -s2);
        }
    }
    if (N(-1, 1, -1) && N(-1, -1, -1)) { /* BACK_TOP_LEFT */
        const double s1 = xy_jx_l * dz + yz_jz_b * dx;
        ADD(-1, 1, -1, s1); ADD(-1, -1, -1, -s1);
    }
    if (N(1, -1, -1) && N(-1, -1, -1)) { /* BACK_DOWN_RIGHT */
        const double s1 = xy_jy_d * dz + xz_jz_b * dy;
        ADD(1, -1, -1, s1); ADD(-1, -1, -1, -s1);
    }
#undef N
#undef ADD
}

int orc_assemble(const mb_monodomain_desc *d, orc_csr *A, int32_t *cells) {
    grid_view G = {d->nx, d->ny, d->nz, d->active};
    const int64_t ng = (int64_t)d->nx * d->ny * d->nz;
    int32_t *row_of = malloc(sizeof(int32_t) * ng);
    if (!row_of) return MB_ERR_NOMEM;
    int32_t n = 0;
    for (int64_t g = 0; g < ng; ++g) row_of[g] = (!d->active || d->active[g]) ? n++ : -1;
    tensor6 *tens = NULL;
    if (d->assembly == MB_ASSEMBLY_ANISOTROPIC) {
        tens = malloc(sizeof(tensor6) * ng);
        if (!tens) { free(row_of); return MB_ERR_NOMEM; }
        for (int k = 0; k < d->nz; ++k) {
            const double th = d->fibre_angle_z ? d->fibre_angle_z[k] : 0.0;
            const tensor6 t = fibre_tensor(th, d->sigma_l, d->sigma_t, d->sigma_n);
            for (int64_t q = 0; q < (int64_t)d->nx * d->ny; ++q) tens[(int64_t)k * d->nx * d->ny + q] = t;
        }
    }
    A->n = n;
    A->row_ptr = malloc(sizeof(int32_t) * ((size_t)n + 1));
    A->col = malloc(sizeof(int32_t) * (size_t)n * 27);
    A->val = malloc(sizeof(double) * (size_t)n * 27);
    if (!A->row_ptr || !A->col || !A->val) {
        free(row_of); free(tens); orc_csr_free(A);
        return MB_ERR_NOMEM;
    }
    const double alpha = alpha_of(d);
    int32_t nnz = 0;
    row27 r;
    A->row_ptr[0] = 0;
    for (int k = 0; k < d->nz; ++k)
        for (int j = 0; j < d->ny; ++j)
            for (int i = 0; i < d->nx; ++i) {
                const int64_t g = i + (int64_t)d->nx * (j + (int64_t)d->ny * k);
                if (row_of[g] < 0) continue;
                if (tens) aniso_row(d, &G, tens, i, j, k, alpha, &r);
                else homogeneous_row(d, &G, i, j, k, alpha, &r);
                if (cells) cells[row_of[g]] = (int32_t)g;
                for (int q = 0; q < r.n; ++q) {
                    if (q > 0 && r.val[q] == 0.0) continue;
                    A->col[nnz] = row_of[r.col[q]];
                    A->val[nnz] = r.val[q];
                    nnz++;
                }
                A->row_ptr[row_of[g] + 1] = nnz;
            }
    free(row_of);
    free(tens);
    return MB_OK;
}

void orc_csr_free(orc_csr *A) {
    free(A->row_ptr);
    free(A->col);
    free(A->val);
    A->row_ptr = A->col = NULL;
    A->val = NULL;
}
