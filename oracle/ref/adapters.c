/*
 * Adapter plugins for the reference MonoAlg3D binary -- TEST INFRASTRUCTURE.
 *
 * The stock plugins cannot express three inputs of the benchmark
 * configurations; these functions express them through the reference's own
 * plugin API, so that the unmodified reference time loop, assembly, CG and
 * cell models run on exactly the tissues the GPU path solves:
 *
 *   initialize_grid_with_mb_cuboid  ([domain] main_function)
 *       the cuboid of initialize_grid_with_cuboid_mesh
 *       (src/domains_library/domain.c:16-38, set_cuboid_domain_mesh in
 *       domain_helpers.c:19-73), then
 *       - a 3-D removed-cell mask read from `mask_file` (nx*ny*nz bytes in
 *         grid order i + nx*(j + ny*k), 0 = removed): the stock
 *         set_plain_fibrosis draws rand() in Hilbert order and
 *         set_fibrosis_from_file is 2-D (domain_helpers.c:689-711,889-965);
 *       - fibres in the xy plane whose angle runs linearly in z from
 *         `fibre_angle_bottom_deg` (z = 0) to `fibre_angle_top_deg` (top),
 *         evaluated at the cell centre, stored in each cell's sigma.fibers
 *         so that anisotropic_sigma_assembly_matrix with fibers_in_mesh=true
 *         assembles per-cell tensors (matrix_assembly.c:389-514; the stock
 *         cuboid has one global f).
 *   set_extra_data_mb_torord_z_layers  ([extra_data] main_function)
 *       the extra data of set_extra_data_mixed_torord_fkatp_epi_mid_endo
 *       (extra_data.c:475-509: set_common_torord_data's current multipliers
 *       and initial states) with the cell types in z-thirds instead of the
 *       stock 45/25/30 % split along x: plane k of nz is ENDO, MID or EPI for
 *       min(2, floor(3 k / nz)) = 0, 1, 2.
 *   save_mb_v_every  ([save_result] main_function, with print_rate=1)
 *       the binary V dump of save_as_text_or_binary (save_mesh.c:248-420 with
 *       binary=true: centre, half sizes and V as 7 doubles per active cell)
 *       written only at iterations that are multiples of `every`, so that
 *       the solver logs the CG of every step (it logs at the save rate,
 *       monodomain_solver.c:763) without a dump at every step.
 *
 * Cells are located by their centres, (i + 1/2) dx etc., as the cuboid
 * builder places them.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/stat.h>

#include "config/domain_config.h"
#include "config/extra_data_config.h"
#include "config/save_mesh_config.h"
#include "config_helpers/config_helpers.h"
#include "domains_library/domain_helpers.h"
#include "extra_data_library/helper_functions.h"
#include "logger/logger.h"

static int cell_index(real_cpu c, real_cpu h) {
    return (int)floor(c / h);
}

SET_SPATIAL_DOMAIN(initialize_grid_with_mb_cuboid) {
    real_cpu start_dx = 0.0, start_dy = 0.0, start_dz = 0.0;
    real_cpu side_length_x = 0.0, side_length_y = 0.0, side_length_z = 0.0;
    GET_PARAMETER_NUMERIC_VALUE_OR_REPORT_ERROR(real_cpu, start_dx, config, "start_dx");
    GET_PARAMETER_NUMERIC_VALUE_OR_REPORT_ERROR(real_cpu, start_dy, config, "start_dy");
    GET_PARAMETER_NUMERIC_VALUE_OR_REPORT_ERROR(real_cpu, start_dz, config, "start_dz");
    GET_PARAMETER_NUMERIC_VALUE_OR_REPORT_ERROR(real_cpu, side_length_x, config, "side_length_x");
    GET_PARAMETER_NUMERIC_VALUE_OR_REPORT_ERROR(real_cpu, side_length_y, config, "side_length_y");
    GET_PARAMETER_NUMERIC_VALUE_OR_REPORT_ERROR(real_cpu, side_length_z, config, "side_length_z");

    char *mask_file = NULL;
    GET_PARAMETER_STRING_VALUE_OR_USE_DEFAULT(mask_file, config, "mask_file");
    real_cpu bottom_deg = NAN, top_deg = NAN;
    GET_PARAMETER_NUMERIC_VALUE_OR_USE_DEFAULT(real_cpu, bottom_deg, config, "fibre_angle_bottom_deg");
    GET_PARAMETER_NUMERIC_VALUE_OR_USE_DEFAULT(real_cpu, top_deg, config, "fibre_angle_top_deg");

    if(!set_cuboid_domain_mesh(the_grid, start_dx, start_dy, start_dz, side_length_x, side_length_y, side_length_z))
        return 0;

    const int nx = (int)lround(side_length_x / start_dx);
    const int ny = (int)lround(side_length_y / start_dy);
    const int nz = (int)lround(side_length_z / start_dz);
    const size_t n = (size_t)nx * ny * nz;

    unsigned char *mask = NULL;
    if(mask_file) {
        FILE *f = fopen(mask_file, "rb");
        if(!f) log_error_and_exit("mask_file %s cannot be opened\n", mask_file);
        mask = malloc(n);
        if(fread(mask, 1, n, f) != n) log_error_and_exit("mask_file %s holds fewer than %zu bytes\n", mask_file, n);
        fclose(f);
    }
    const int rotate = !isnan(bottom_deg) && !isnan(top_deg);
    size_t removed = 0;

    FOR_EACH_CELL(the_grid) {
        if(!cell->active) continue;
        const int i = cell_index(cell->center.x, start_dx);
        const int j = cell_index(cell->center.y, start_dy);
        const int k = cell_index(cell->center.z, start_dz);
        if(i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz)
            log_error_and_exit("active cell outside the %d x %d x %d cuboid\n", nx, ny, nz);
        if(mask && !mask[(size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)]) {
            cell->active = false;
            removed++;
        }
        if(rotate) {
            /* the same operations, in the same order, as the GPU workload's
               angles: (bottom + (top - bottom) (k + 1/2) / nz) (pi / 180) */
            const real_cpu t = ((real_cpu)k + 0.5) / nz;
            const real_cpu th = (bottom_deg + (top_deg - bottom_deg) * t) * (M_PI / 180.0);
            struct fiber_coords *fc = &cell->sigma.fibers;
            fc->f[0] = cos(th); fc->f[1] = sin(th); fc->f[2] = 0.0;
            fc->s[0] = -sin(th); fc->s[1] = cos(th); fc->s[2] = 0.0;
            fc->n[0] = 0.0; fc->n[1] = 0.0; fc->n[2] = 1.0;
        }
    }
    free(mask);
    log_info("mb cuboid: %d x %d x %d cells, %zu removed by the mask, fibres %s\n", nx, ny, nz, removed,
             rotate ? "rotating in z" : "from the assembly section");
    return 1;
}

SET_EXTRA_DATA(set_extra_data_mb_torord_z_layers) {
    uint32_t num_active_cells = the_grid->num_active_cells;
    struct cell_node **ac = the_grid->active_cells;

    real_cpu start_dz = 0.0, side_length_z = 0.0;
    GET_PARAMETER_NUMERIC_VALUE_OR_REPORT_ERROR(real_cpu, start_dz, config, "start_dz");
    GET_PARAMETER_NUMERIC_VALUE_OR_REPORT_ERROR(real_cpu, side_length_z, config, "side_length_z");
    const int nz = (int)lround(side_length_z / start_dz);

    struct extra_data_for_torord *extra_data = set_common_torord_data(config, num_active_cells);

    for(uint32_t i = 0; i < num_active_cells; i++) {
        const int k = cell_index(ac[i]->center.z, start_dz);
        int t = (3 * k) / nz;
        if(t > 2) t = 2;
        extra_data->transmurality[i] = (real)t;
    }

    SET_EXTRA_DATA_SIZE(sizeof(struct extra_data_for_torord));
    return (void *)extra_data;
}

SAVE_MESH(save_mb_v_every) {
    int every = 50;
    GET_PARAMETER_NUMERIC_VALUE_OR_USE_DEFAULT(int, every, config, "every");
    char *output_dir = NULL;
    GET_PARAMETER_STRING_VALUE_OR_REPORT_ERROR(output_dir, config, "output_dir");
    if(every <= 0 || time_info->iteration % every != 0) return;
    mkdir(output_dir, 0755);
    char path[4096];
    snprintf(path, sizeof path, "%s/V_it_%d.bin", output_dir, time_info->iteration);
    FILE *f = fopen(path, "wb");
    if(!f) log_error_and_exit("cannot write %s\n", path);
    const uint32_t n = the_grid->num_active_cells;
    struct cell_node **ac = the_grid->active_cells;
    for(uint32_t i = 0; i < n; i++) {
        const double rec[7] = {ac[i]->center.x, ac[i]->center.y, ac[i]->center.z, ac[i]->discretization.x / 2.0,
                               ac[i]->discretization.y / 2.0, ac[i]->discretization.z / 2.0, ac[i]->v};
        fwrite(rec, sizeof(double), 7, f);
    }
    fclose(f);
}
