/* Host assembly of the monodomain diffusion operator (C). */
#ifndef MB_ASSEMBLY_H
#define MB_ASSEMBLY_H

#include "monoalg3d_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mb_assembly_out {
    int kind;                 /* 0 constant 7-point, 1 per-face 7-point, 2 class table */
    double cx, cy, cz;        /* kind 0 */
    double *fx, *fy, *fz;     /* kind 1, nx*ny*nz each */
    double *table;            /* kind 2, nz * 9 * 27 */
} mb_assembly_out;

/* Conductivity tensor of one cell and whether it exists (active). */
typedef struct mb_nb_sigma {
    int exists;
    double x, y, z, xy, xz, yz;
} mb_nb_sigma;

int  mb_assemble(const mb_monodomain_desc *d, mb_assembly_out *out);
void mb_assembly_free(mb_assembly_out *out);

/* One row of anisotropic_sigma_assembly_matrix: nb[27] indexed by
 * (dz+1)*9 + (dy+1)*3 + (dx+1), centre at 13.  row[27] receives the matrix
 * coefficients per neighbour offset (row[13] = diagonal, alpha included). */
void mb_aniso_row(const mb_nb_sigma nb[27], double dx, double dy, double dz, double alpha, double row[27]);

/* D = (sigma_l - sigma_t) f f^T + sigma_t I  (calc_tensor2) or
 * D = sigma_l f f^T + sigma_t s s^T + sigma_n n n^T (calc_tensor). */
void mb_fibre_tensor(const double f[3], const double s[3], const double n[3], double sigma_l, double sigma_t,
                     double sigma_n, double D[3][3]);

double mb_alpha(double beta, double cm, double dt, double dx, double dy, double dz);
double mb_tt2006_default_state(int s);
double mb_torord_default_state(int celltype, int s);
double mb_torord_endo_default_state(int gpu_build, int s);
int mb_monodomain_uses_graphs(mb_monodomain *m);

#ifdef __cplusplus
}
#endif

#endif
