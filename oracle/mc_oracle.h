/* mc_oracle.h - CPU restatement of the reference's render hot path.
 *
 * TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg (and its reference arm when the reference build is absent)
 * call into this library; the product (libmcpt.so) never does.
 *
 * Parity: pinned against the unmodified reference compiled in oracle/_ref
 * (host-side Morton codes, sort order, bounds and camera bit-exact; device-side
 * topology, hits and images through fixtures in tests/golden/ that
 * tests/golden/make_golden.py generates by running that build on a B200).
 */
#ifndef MC_ORACLE_H
#define MC_ORACLE_H
#include <stdint.h>
#include "mc_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* finalizeScene + main()'s std::sort (PT:1930-1987, 4223-4233). perm[k] is the
 * reference-list position (spheres first) of the k-th sorted primitive. */
int orc_finalize_sort(const mc_triangle* tris, int nt, const mc_sphere* sph, int ns, uint32_t* codes_ref_order,
                      uint32_t* sorted_codes, int32_t* perm, mc_aabb* bounds_ref_order, mc_aabb* scene_bounds);

/* Karras hierarchy + leaves + refit (PT:1063-1090, 1337-1447) on sorted codes.
 * internal: n-1 nodes, leaves: n nodes (reference layout). */
int orc_build(const uint32_t* sorted_codes, const int32_t* perm, const mc_aabb* bounds_ref_order, int n, int ns,
              mc_bvh_node* internal, mc_bvh_node* leaves);

/* Max leaf depth (edges from the root). */
int orc_depth(const mc_bvh_node* internal, const mc_bvh_node* leaves, int n);

/* Ray set through the reference's traversal order (PT:1092-1321). rays: SoA 7*nr.
 * mode 0 closest -> hits; mode 1 any hit within tmax -> occluded. Double = 0
 * evaluates in float (IEEE), 1 in double. */
int orc_trace(const mc_bvh_node* internal, const mc_bvh_node* leaves, const int32_t* leaf_types, int n,
              const mc_triangle_hot* hot, const mc_sphere* sph, const float* rays, int nr, int mode, const float* tmax,
              mc_packed_hit* hits, int32_t* occluded, int threads);

/* A scene prepared for rendering: the reference's finalize, sort and LBVH on
 * the host, its light list, and the environment map with its sampling tables
 * (buildEnvironmentSamplingTables, PT:370-385). env_rgba may be NULL. */
void* orc_scene_create(const mc_triangle* tris, int nt, const mc_sphere* sph, int ns, const float* env_rgba, int env_w,
                       int env_h, float env_intensity, float env_rotation);
void orc_scene_destroy(void* scene);

/* Path tracer over a pixel rectangle [x0,x1) x [y0,y1) of a W x H image, with
 * the reference's integrator (PT:2900-3059 / 3342-3755) and counter-based Philox
 * draws keyed by (seed, pixel, sample). accum: W*H*3 doubles, added into.
 * stats (may be NULL): [0] extend rays, [1] shadow rays. */
int orc_render(void* scene, const mc_camera* cam, int W, int H, int spp, int first_sample, int max_depth, uint64_t seed,
               int use_double, int disable_clamp, int x0, int y0, int x1, int y1, int threads, double* accum,
               double* stats);

/* Guiding MLP in FP64 (mc_guide_oracle.cpp). params: MC_GUIDE_PARAM_COUNT
 * doubles; lo/inv: the guide box's low corner and 1/extent (3 floats each).
 * Forward: n queries (6 floats) -> n x 40 mixtures. Loss/gradient: n records
 * (10 floats) -> gradient (PARAM_COUNT doubles) and the loss. flags: bit 0
 * rounds the values the tensor-core kernels round; bit 1 anchors the lobes
 * (every raw mean offset by 1.5 x the direction input, mc_guide_config.
 * anchor_lobes); bit 2 with bit 1 uses -1.5 (MC_GUIDE_DIR_RAY guides). */
int orc_guide_forward(const double* params, const float* queries, int n, const float* lo, const float* inv,
                      int flags, double* mix);
int orc_guide_loss_grad(const double* params, const float* records, int n, const float* lo, const float* inv,
                        int flags, double* grad, double* loss);

/* Philox-4x32-10 block (known-answer checks). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

#ifdef __cplusplus
}
#endif
#endif
