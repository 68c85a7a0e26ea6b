/*
 * fot_oracle.h -- CPU oracle for the indirect-increment loops.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker, never the thing
 * measured or shipped: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py may load it.  The product path
 * (cuda_fot_b200/libfot.so) neither links nor calls it.
 *
 * It restates, in plain C, the reference's serial loop driver
 * (problem.hpp:342-380, Problem::stepCPUCellCentred / loopCPUCellCentred) and
 * the five StepSeq kernels with their user functors:
 *   res_calc  kernels/res_calc.hpp:29-89      + kernels/res_calc_func.hpp:9-60
 *   mini_aero kernels/mini_aero.hpp:43-111    + kernels/mini_aero_func.hpp:11-85
 *                                             + kernels/mini_aero_utils.hpp:6-373
 *   lulesh    kernels/lulesh.hpp:23-58        + kernels/lulesh_func.hpp:11-37
 *                                             + kernels/lulesh_utils.hpp:4-200
 *   volna     kernels/volna.hpp:30-75         + kernels/volna_func.hpp:16-35
 *   getacc    kernels/getacc_scatter.hpp:29-75 + kernels/getacc_scatter_func.hpp:18-96
 * with the data bindings of the app drivers' initProblem
 * (res_calc.cu:10-28, mini_aero.cu:10-24, lulesh.cu:10-24, volna.cu:11-27,
 * getacc.cu:11-26).  Every floating-point operation is written in the same
 * order as the reference and the library is compiled with
 * -ffp-contract=off, so on the same inputs the serial loop here is
 * bit-identical to the reference's (pinned by tests/golden, generated from the
 * reference's own compiled serial loop).
 *
 * Beyond the reference it adds:
 *   - orc_replay_hier: the CPU replay of a hierarchical-colour plan (block
 *     colours in order, inside a block a zeroed cache summed in thread-colour
 *     order, then out += cache), the bit-exact target for the coloured GPU run
 *     (the order of res_calc.hpp:319-358);
 *   - orc_check_plan: exact integer checks of a plan;
 *   - orc_point_graph / orc_reorder_inverse: the point-to-point CSR graph of a
 *     mapping (reorder.hpp:33-132, 177-202), pinned by the reference's Catch KAT;
 *   - orc_airfoil_run: the Airfoil solver iteration the engine runs around
 *     res_calc (its other loops are not in the reference: pinned instead to
 *     an independent Python statement in the tests).
 */
#ifndef FOT_ORACLE_H
#define FOT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORC_RES_CALC = 0,
  ORC_MINI_AERO = 1,
  ORC_LULESH = 2,
  ORC_VOLNA = 3,
  ORC_GETACC = 4
};

/* Serial loop in cell order, `iters` times.  point_data[k] is the k-th point
 * dataset in the problem layout (AOS when soa == 0, SOA otherwise);
 * cell_data[j] is always SOA with stride n_cells.  point_data[0] (and for
 * lulesh cell_data[1], "determ") are updated in place.  maps[k] is the AOS
 * cell-to-point mapping k (n_cells x mesh_dim).  Returns 0 on success. */
int orc_loop_serial(int loop, int soa, uint32_t n_cells,
                    const uint32_t *n_points, const uint32_t *const *maps,
                    void *const *point_data, void *const *cell_data,
                    uint32_t iters);

/* Hierarchical-colour plan in execution order (arrays as exported by the
 * engine's fot_plan_export): blocks are stored colour-major; within a block,
 * positions are sorted by thread colour. */
typedef struct orc_plan {
  uint32_t n_cells, n_blocks, n_colours, mesh_dim;
  const uint32_t *colour_offsets; /* n_colours+1, block index where a colour starts */
  const uint32_t *block_start;    /* n_blocks+1, first position of each block */
  const uint32_t *cell_id;        /* n_cells, position -> original cell */
  const uint8_t *tcol;            /* n_cells, thread colour of each position */
  const uint8_t *block_ntcol;     /* n_blocks, thread colours used by a block */
  const uint32_t *pts_off;        /* n_blocks+1, offsets into pts (written set) */
  const uint32_t *pts;            /* unique written points of each block, ascending */
  const uint16_t *lidx;           /* mesh_dim x n_cells (SOA), local index into the block's pts */
} orc_plan;

/* CPU replay of the coloured plan.  Same arguments as orc_loop_serial. */
int orc_replay_hier(int loop, int soa, uint32_t n_cells,
                    const uint32_t *n_points, const uint32_t *const *maps,
                    void *const *point_data, void *const *cell_data,
                    uint32_t iters, const orc_plan *plan);

/* The Airfoil solver iteration the engine runs around res_calc
 * (fot_airfoil_run; not part of the reference, which drives res_calc alone):
 * save_soln, then twice { adt_calc, res_calc, bres_calc, update }, with the
 * same operations in the same order as the engine's kernels.  point_data are
 * res_calc's (res 0, x 1, q 2, adt 3) in the problem layout; res_calc runs in
 * serial edge order when P is NULL, else replays P's colour order.  The
 * boundary edges add in edge order; rms = sqrt(sum of squared updates /
 * cells) of the last iteration's second stage, summed in cell order. */
typedef struct orc_airfoil {
  const uint32_t *cell_to_node;  /* n_cells x 4 */
  uint32_t n_bedges;
  const uint32_t *bedge_to_node; /* n_bedges x 2 */
  const uint32_t *bedge_to_cell;
  const int32_t *bound;
  double qinf[4];
  double cfl;
} orc_airfoil;
int orc_airfoil_run(int soa, uint32_t n_edges, const uint32_t *n_points,
                    const uint32_t *const *maps, void *const *point_data,
                    const orc_airfoil *A, uint32_t iters, const orc_plan *P,
                    double *rms);

/* Exact checks of a plan against mapping 0 (n_cells x mesh_dim) and the block
 * size.  Returns 0 when valid, otherwise a nonzero code naming the first
 * failed check (see fot_oracle.c) and writes a message into err. */
int orc_check_plan(const orc_plan *plan, const uint32_t *map0,
                   uint32_t n_points0, uint32_t block_size, char *err,
                   uint32_t err_len);

/* 1 if perm is a bijection of [0, n), else 0. */
int orc_is_permutation(const uint32_t *perm, uint32_t n);

/* Point-to-point CSR graph of a mapping: two points are adjacent when a cell
 * holds both (reorder.hpp:38-78).  indices has n_points+1 entries; endpoints
 * must have room for n_cells*dim*(dim-1) entries; rows are sorted ascending.
 * Returns the number of arcs. */
uint32_t orc_point_graph(uint32_t n_points, uint32_t n_cells, uint32_t dim,
                         const uint32_t *map, uint32_t *indices,
                         uint32_t *endpoints);

/* Bandwidth and profile of mapping 0 under its current numbering:
 * bandwidth = max over cells of (max point - min point); profile = sum over
 * points p of (p - smallest neighbour of p) for neighbours below p. */
void orc_bandwidth_profile(uint32_t n_points, uint32_t n_cells, uint32_t dim,
                           const uint32_t *map, uint64_t *bandwidth,
                           uint64_t *profile);

#ifdef __cplusplus
}
#endif
#endif
