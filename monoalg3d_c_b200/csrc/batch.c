/* Batches of independent tissues (host, C).
 *
 * Many small tissues -- 1-D cables and 2-D sheets of uneven size -- are
 * solved as one: mb_batch_pack places them side by side in one 2-D atlas
 * grid, each surrounded by removed cells, so that no face couples two
 * tissues.  The atlas is then an ordinary tissue with removed cells: one ODE
 * launch advances every cell of every tissue, one persistent CG launch solves
 * every tissue's implicit diffusion system, and the whole step is one CUDA
 * graph replay.  Per-tissue parameters (conductance scalings, stimulus
 * regions) become per-cell arrays of the atlas.
 *
 * The stacked system is block diagonal, one block per tissue; CG on it stops
 * when the summed r.r reaches the tolerance, so every tissue's own residual
 * is at least as small as its stand-alone solve would leave it.
 *
 * Packing: shelves, tallest tissue first.  Tissues are sorted by height (then
 * width, then index), laid left to right with one removed column between
 * them; a shelf is as tall as its first tissue and shelves are separated by
 * one removed row.  The atlas width is the smallest multiple of 32 at least
 * sqrt(1.05 x the area with gaps) and at least the widest tissue + 2.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "monoalg3d_b200.h"

typedef struct pack_item { int idx, nx, ny; } pack_item;

static int by_height(const void *a, const void *b) {
    const pack_item *p = (const pack_item *)a, *q = (const pack_item *)b;
    if (p->ny != q->ny) return q->ny - p->ny;
    if (p->nx != q->nx) return q->nx - p->nx;
    return p->idx - q->idx;
}

int mb_batch_pack(int n, const int *nx, const int *ny, int *atlas_nx, int *atlas_ny, int *x0, int *y0) {
    if (n <= 0 || !nx || !ny || !atlas_nx || !atlas_ny || !x0 || !y0) return MB_ERR_ARG;
    pack_item *it = (pack_item *)malloc(sizeof(pack_item) * (size_t)n);
    if (!it) return MB_ERR_NOMEM;
    double area = 0.0;
    int widest = 0;
    for (int i = 0; i < n; ++i) {
        if (nx[i] <= 0 || ny[i] <= 0) { free(it); return MB_ERR_ARG; }
        it[i].idx = i;
        it[i].nx = nx[i];
        it[i].ny = ny[i];
        area += (double)(nx[i] + 1) * (double)(ny[i] + 1);
        if (nx[i] > widest) widest = nx[i];
    }
    qsort(it, (size_t)n, sizeof(pack_item), by_height);
    int W = (int)ceil(sqrt(1.05 * area));
    if (W < widest + 2) W = widest + 2;
    W = (W + 31) & ~31;
    int x = 1, y = 1, shelf_h = 0;
    for (int q = 0; q < n; ++q) {
        if (x + it[q].nx + 1 > W) {          /* next shelf */
            y += shelf_h + 1;
            x = 1;
            shelf_h = 0;
        }
        x0[it[q].idx] = x;
        y0[it[q].idx] = y;
        x += it[q].nx + 1;
        if (it[q].ny > shelf_h) shelf_h = it[q].ny;
    }
    *atlas_nx = W;
    *atlas_ny = y + shelf_h + 1;
    free(it);
    return MB_OK;
}
