/*
 * Prints the cells of a reference MonoAlg3D grid in the order of its linked
 * list (the Hilbert order in which save_simulation_state writes them and in
 * which order_grid_cells numbers the active ones) -- TEST INFRASTRUCTURE.
 *
 *   hilbert_probe cube <side_cells> <levels>
 *       a cube of side_cells x 100 um refined `levels` times
 *       (initialize_and_construct_grid + refine_grid, grid.c / grid_refinement.c)
 *   hilbert_probe cuboid <nx> <ny> <nz>
 *       the cuboid of set_cuboid_domain_mesh (domain_helpers.c:19-73) at 100 um
 *
 * Output: one line per cell "i j k active" (cell indices from the centres).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#include "alg/grid/grid.h"
#include "domains_library/domain_helpers.h"

int main(int argc, char **argv) {
    if(argc < 4) return 2;
    struct grid *g = new_grid();
    const double h = 100.0;
    if(!strcmp(argv[1], "cube")) {
        const double side = atof(argv[2]) * h;
        initialize_and_construct_grid(g, POINT3D(side, side, side));
        refine_grid(g, atoi(argv[3]));
    } else {
        if(argc < 5) return 2;
        if(!set_cuboid_domain_mesh(g, h, h, h, atof(argv[2]) * h, atof(argv[3]) * h, atof(argv[4]) * h)) return 1;
    }
    FOR_EACH_CELL(g) {
        printf("%d %d %d %d\n", (int)floor(cell->center.x / h), (int)floor(cell->center.y / h),
               (int)floor(cell->center.z / h), cell->active ? 1 : 0);
    }
    return 0;
}
