/*
 * svsflow.h - C ABI of the B200 (sm_100a) 3D TV-L1 optical-flow and mask-propagation library
 * (libsvsflow.so).
 *
 * It replaces the reference's pybind module `opticalFlow_cuda_ext.opticalFlow`
 * (svs/src/bindings.cpp:16-192, 3D subset) and the per-pair solver loop of
 * svs/modules/flow/tvl13d.py:122-255. All pointers are DEVICE pointers unless a comment says
 * otherwise; sizes are element counts; every call is asynchronous on the given stream
 * (NULL = the legacy default stream, which is where the reference launched its kernels).
 *
 * Layouts are the reference's: C-order, components last.
 *   scalar field  [NZ,NY,NX]          vector field [NZ,NY,NX,3]
 *   matrix field  [NZ,NY,NX,3,3]      (row = flow component, column = derivative x,y,z)
 *   CNN volume    [B,C,NZ,NY,NX]      flow for CNN warp [B,NZ,NY,NX,3]
 * Vector component 0 is x (fastest axis), 1 is y, 2 is z.
 *
 * Errors: every entry point returns an svs_status. On failure, svs_last_error() returns a
 * thread-local message. The reference raised c10::Error (TORCH_CHECK / CHECK_INPUT,
 * svs/src/coreDefines.h:10-12) and ignored launch errors (svs/src/cudaDebug.cuh:15-27); here
 * argument errors and launch errors are both reported.
 */
#ifndef SVSFLOW_H_
#define SVSFLOW_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* svs_stream_t; /* == cudaStream_t */

typedef enum {
  SVS_OK = 0,
  SVS_ERR_INVALID_ARG = 1,
  SVS_ERR_OUT_OF_MEMORY = 2,
  SVS_ERR_LAUNCH = 3,
  SVS_ERR_TIMEOUT = 4,
  SVS_ERR_UNSUPPORTED = 5,
  SVS_ERR_CUDA = 6
} svs_status;

/* svs/src/boundary.cuh:13-21 */
enum { SVS_BOUNDARY_NEAREST = 0, SVS_BOUNDARY_MIRROR = 1, SVS_BOUNDARY_REFLECT = 2 };
/* svs/src/coreDefines.h:94-100 */
enum { SVS_INTERPOLATE_NEAREST = 0, SVS_INTERPOLATE_LINEAR = 1, SVS_INTERPOLATE_CUBIC_HERMITESPLINE = 2 };
/* storage precision of the fused solver's iteration state (arithmetic is always FP32):
 * all fields F32; all fields BF16 or FP16; or the flow u in F32 with the dual field, the tensor
 * D and the linearisation (rho_c, warped gradient) in BF16 / FP16. */
enum {
  SVS_STORAGE_F32 = 0,
  SVS_STORAGE_BF16 = 1,
  SVS_STORAGE_F16 = 2,
  SVS_STORAGE_BF16_FLOW32 = 3,
  SVS_STORAGE_F16_FLOW32 = 4
};

const char* svs_last_error(void);
int svs_version(void);

/* ---------------------------------------------------------------------------------------------
 * Per-operator entry points (one reference op each). h = mesh spacing L/(N-1) per axis.
 * ------------------------------------------------------------------------------------------- */

/* Nabla3D_CD.forward (svs/src/differentialOps.h:82-85; kernels differentialOps.cu:540-655)
 * and .forwardVectorField (:90-93; differentialOps.cu:782-907): central-difference gradient of
 * each of the C components of b [NZ,NY,NX,C] into out [NZ,NY,NX,C,3]. C = 1 is .forward. */
svs_status svs_nabla3d_forward(const float* b, int nz, int ny, int nx, int C, float hz, float hy,
                               float hx, int boundary, float* out, svs_stream_t stream);

/* Nabla3D_CD.backward / .backwardVectorField (differentialOps.h:86-89, :94-97; kernels
 * differentialOps.cu:658-779, :909-1039): adjoint of the gradient, p [NZ,NY,NX,C,3] -> out
 * [NZ,NY,NX,C]. */
svs_status svs_nabla3d_backward(const float* p, int nz, int ny, int nx, int C, float hz, float hy,
                                float hx, int boundary, float* out, svs_stream_t stream);

/* AnisotropicNabla3D.computeTangentVecs (anisotropicDifferentialOps.h:414-420; kernel
 * anisotropicDifferentialOps.cu:89-141): g [n,3] -> s [n], normals, t1, t2 [n,3]. */
svs_status svs_aniso3d_tangents(const float* g, int64_t n, float alpha, float beta, float* s,
                                float* normals, float* t1, float* t2, svs_stream_t stream);

/* AnisotropicNabla3D.forwardVectorField / .backwardVectorField (identical in the reference,
 * anisotropicDifferentialOps.h:422-444; kernel anisotropicDifferentialOps.cu:143-175):
 * out[c][d] = s (n.in_c) n[d] + (t1.in_c) t1[d] for in/out [n,3,3]. t2 is accepted and unused
 * (its factor is never accumulated in the reference). */
svs_status svs_aniso3d_apply(const float* in, int64_t n, const float* s, const float* normals,
                             const float* t1, const float* t2, float* out, svs_stream_t stream);

/* TVL1OF3D_proxPrimal (opticalFlowOps.h:111-120; kernel opticalFlowOps.cu:123-175). */
svs_status svs_tvl1_prox_primal(const float* primal, int64_t n, float tau, float weight_matching,
                                const float* rho, const float* i1w_grad, float* out,
                                svs_stream_t stream);

/* TVL1OF3D_proxDual (opticalFlowOps.h:123-129; kernel opticalFlowOps.cu:179-208). sigma is
 * accepted and unused, as in the reference. */
svs_status svs_tvl1_prox_dual(const float* dual, int64_t n, float sigma, float weight_tv,
                              float* out, svs_stream_t stream);

/* Warping3D.forward / .forwardVectorField (warpingOps.h:87-116; kernels warpingOps.cu:572-660
 * and their nearest/trilinear siblings): out(x) = u(x + phi(x)) for u [NZ,NY,NX,C],
 * phi [NZ,NY,NX,3]. */
svs_status svs_warp3d(const float* u, int nz, int ny, int nx, int C, const float* phi, float hz,
                      float hy, float hx, int interpolation, int boundary, float* out,
                      svs_stream_t stream);

/* Warping3D.backward (warpingOps.h:103-108; kernels warpingOps.cu:172-200, :384-412, :598-630;
 * interpolation_*.cuh 3D backward helpers): gradients of sum(grad_out * warp(u, phi)) with
 * respect to u [NZ,NY,NX] (scattered with atomic adds onto the folded stencil nodes, as the
 * reference does) and phi [NZ,NY,NX,3] (the derivative of the interpolant at the sample point
 * divided by h; zero for nearest). grad_u and grad_phi are overwritten. Scalar fields only, as
 * in the reference. */
svs_status svs_warp3d_backward(const float* u, int nz, int ny, int nx, const float* phi,
                               const float* grad_out, float hz, float hy, float hx,
                               int interpolation, int boundary, float* grad_u, float* grad_phi,
                               svs_stream_t stream);

/* WarpingCNN3D.forward (warpingOpsCNN.h:240-263; kernel warpingOpsCNN.cu:97-128):
 * out[b,c] = m[b,c](x + phi[b](x)) for m [B,C,NZ,NY,NX], phi [B,NZ,NY,NX,3]. */
svs_status svs_warp_cnn3d(const float* m, int B, int C, int nz, int ny, int nx, const float* phi,
                          float hz, float hy, float hx, int interpolation, int boundary,
                          float* out, svs_stream_t stream);

/* Prolongation3D.forward / .forwardVectorField / .forwardMatrixField (prolongationOps.h:79-107;
 * kernels prolongationOps.cu:533-625): resample a C-component field from mesh (n*, L*) to mesh
 * (t*, tL*); target node i samples the source at (i*h_t)*L_s/L_t. */
svs_status svs_prolongate3d(const float* u, int nz, int ny, int nx, int C, float lz, float ly,
                            float lx, int tz, int ty, int tx, float tlz, float tly, float tlx,
                            int interpolation, int boundary, float* out, svs_stream_t stream);

/* apply_gaussian_blur3d (svs/utils/flow_utils.py:94-112): zero-padded 3D correlation of
 * in [NZ,NY,NX] with a (2r+1)^3 kernel given in HOST memory (weights_host, float32). */
svs_status svs_gauss_blur3d(const float* in, int nz, int ny, int nx, const float* weights_host,
                            int r, float* out, svs_stream_t stream);

/* apply_median_filter (svs/utils/flow_utils.py:115-132): ks^3 median (ks = 3 or 5) of each
 * component of in [NZ,NY,NX,C], scipy 'reflect' boundary. Replaces the reference's host round
 * trip through scipy. */
svs_status svs_median3d(const float* in, int nz, int ny, int nx, int C, int ks, float* out,
                        svs_stream_t stream);

/* FP64 forms of the per-operator entry points above: the same operators, arguments and
 * semantics on double arrays, with double scalars (the reference dispatches float and double,
 * AT_DISPATCH_FLOATING_TYPES in the .cu files of svs/src). Used by the double-precision drop-in operators and
 * the FP64 run of the plain solver on the GPU. */
svs_status svs_nabla3d_forward_f64(const double* b, int nz, int ny, int nx, int C, double hz, double hy,
                                   double hx, int boundary, double* out, svs_stream_t stream);
svs_status svs_nabla3d_backward_f64(const double* p, int nz, int ny, int nx, int C, double hz, double hy,
                                    double hx, int boundary, double* out, svs_stream_t stream);
svs_status svs_aniso3d_tangents_f64(const double* g, int64_t n, double alpha, double beta, double* s,
                                    double* normals, double* t1, double* t2, svs_stream_t stream);
svs_status svs_aniso3d_apply_f64(const double* in, int64_t n, const double* s, const double* normals,
                                 const double* t1, const double* t2, double* out, svs_stream_t stream);
svs_status svs_tvl1_prox_primal_f64(const double* primal, int64_t n, double tau, double weight_matching,
                                    const double* rho, const double* i1w_grad, double* out, svs_stream_t stream);
svs_status svs_tvl1_prox_dual_f64(const double* dual, int64_t n, double sigma, double weight_tv, double* out,
                                  svs_stream_t stream);
svs_status svs_warp3d_f64(const double* u, int nz, int ny, int nx, int C, const double* phi, double hz,
                          double hy, double hx, int interpolation, int boundary, double* out, svs_stream_t stream);
svs_status svs_warp3d_backward_f64(const double* u, int nz, int ny, int nx, const double* phi,
                                   const double* grad_out, double hz, double hy, double hx, int interpolation,
                                   int boundary, double* grad_u, double* grad_phi, svs_stream_t stream);
svs_status svs_warp_cnn3d_f64(const double* m, int B, int C, int nz, int ny, int nx, const double* phi,
                              double hz, double hy, double hx, int interpolation, int boundary, double* out,
                              svs_stream_t stream);
svs_status svs_prolongate3d_f64(const double* u, int nz, int ny, int nx, int C, double lz, double ly,
                                double lx, int tz, int ty, int tx, double tlz, double tly, double tlx,
                                int interpolation, int boundary, double* out, svs_stream_t stream);
svs_status svs_gauss_blur3d_f64(const double* in, int nz, int ny, int nx, const double* weights_host, int r,
                                double* out, svs_stream_t stream);
svs_status svs_median3d_f64(const double* in, int nz, int ny, int nx, int C, int ks, double* out,
                            svs_stream_t stream);

/* ---------------------------------------------------------------------------------------------
 * Fused solver: TVL13DOpticalFlow.compute (svs/modules/flow/tvl13d.py:122-162) for a batch of
 * independent frame pairs. Every pair is solved from zero flow at the coarsest level (the
 * reference's warm start is overwritten when num_scales > 1, tvl13d.py:150, 158).
 * ------------------------------------------------------------------------------------------- */
typedef struct svs_tvl1_params {
  int num_scales;            /* tvl13d.py:55 */
  int max_warps;             /* :56 */
  int max_outer_iterations;  /* :57 */
  float weight_matching;     /* :58 (lambda of the L1 data term) */
  float weight_tv;           /* :59 (radius of the dual ball) */
  int primaldual_algorithm_type; /* :60 (1: fixed steps, 2: accelerated schedule) */
  double sigma, tau, theta, gamma; /* :61 (theta is never used for extrapolation) */
  int use_anisotropic_diff;  /* :62 */
  float alpha, beta;         /* :63 */
  int use_gaussian_blur;     /* :64 */
  float gaussian_blur_sigma; /* :65 */
  int interpolation;         /* :68 (solver kernels require CUBIC_HERMITESPLINE) */
  int boundary;              /* :68 */
  int length_type;           /* 0 = numDofs (L = N-1, h = 1), 1 = fixed lengths below */
  float length_z, length_y, length_x;
  int median_kernel;         /* 0 = off, else the processor's post-filter size (processor.py:116) */
  int storage;               /* SVS_STORAGE_* for the iteration state */
} svs_tvl1_params;

typedef struct svs_pair_desc {
  int nz, ny, nx;
  const float* I0; /* [nz,ny,nx] fixed frame (processor.py:111: img[t_{j+1}]) */
  const float* I1; /* [nz,ny,nx] moving frame (processor.py:112: img[t_j]) */
  float* u_out;    /* [nz,ny,nx,3] flow */
  float* p_out;    /* [nz,ny,nx,3,3] dual field, or NULL */
  const float* u_init; /* [nz,ny,nx,3] warm start or NULL; used only when num_scales == 1 */
  const float* p_init; /* [nz,ny,nx,3,3] warm start or NULL; used only when num_scales == 1 */
} svs_pair_desc;

typedef struct svs_plan svs_plan;

/* Create a plan for a batch of up to max_pairs pairs whose level-0 sizes are listed in
 * dims[3*i .. 3*i+2] (nz, ny, nx). The plan owns all device state (pyramids, dual fields,
 * linearisation) and one CUDA graph of the whole batched solve, built on first use. */
svs_status svs_tvl1_plan_create(const svs_tvl1_params* params, int num_pairs,
                                const int* dims_host, svs_plan** plan);
svs_status svs_tvl1_plan_destroy(svs_plan* plan);
/* Bytes of device memory the plan holds. */
size_t svs_tvl1_plan_device_bytes(const svs_plan* plan);
/* Select the iterate-kernel variant (0 = automatic) for later solves; SVS_ERR_INVALID_ARG for an
 * unknown id. Variants 1-5 are TMA pipelines (tile x prefetch distance: 32x8/2, 32x8/3, 64x4/2,
 * 16x16/2, 32x16/2), 6-8 plain-load forms (32x8, 32x4, 16x16), 9-33 split-role TMA pipelines
 * (interior, halo-row and halo-column lanes in separate warps; 21-24 synchronise with mbarriers
 * and a producer warp instead of a block-wide barrier per plane; 25-33 are placement and
 * schedule options of the 40x8, 32x16 and 16x16 shapes for FP32 and f16-flow32 storage, other
 * storages report SVS_ERR_UNSUPPORTED for them; svs_tvl1_tile_info gives each shape). Used by the
 * autotuner. */
svs_status svs_tvl1_plan_set_tile(svs_plan* plan, int tile_id);
/* Same for one pyramid level only (0 = fall back to the plan-wide choice). */
svs_status svs_tvl1_plan_set_level_tile(svs_plan* plan, int level, int tile_id);
/* Same for one pair at one level (0 = the level's variant). Pairs of a level that ask for another
 * variant than the level's form a group per variant; the groups run concurrently (parallel
 * branches of the solve's graph). Used by the autotuner to pick variants per size class. */
svs_status svs_tvl1_plan_set_pair_tile(svs_plan* plan, int level, int pair, int tile_id);
/* Number of z chunks each column tile of a level is split into (0 = the automatic choice: the
 * wave model for the TMA-pipeline variants). More chunks mean more CTAs, each marching fewer
 * planes. Used by the autotuner. */
svs_status svs_tvl1_plan_set_level_chunks(svs_plan* plan, int level, int chunks);
int svs_tvl1_num_tiles(void);

/* Residuals. With record != 0 every later solve logs, after each warp of each level, the
 * root-mean-square change of each pair's flow over that warp, sqrt(sum (u_w - u_{w-1})^2 / 3N),
 * reduced in FP64. With stop_tol > 0 a pair whose change falls below stop_tol skips the remaining
 * warps of that level (its flow is final for the level); stop_tol > 0 needs an even
 * max_outer_iterations. The reference computes per-iteration norms of the changes and never uses
 * them (svs/modules/flow/tvl13d.py:240-253), always running every warp: record = 0 and
 * stop_tol = 0 (the default) keep its schedule. Allocates the log and snapshot buffers. */
svs_status svs_tvl1_plan_set_residuals(svs_plan* plan, int record, float stop_tol);
/* Residual log of the last solve into out_host[(pair * levels + level) * max_warps + warp]
 * (level 0 = finest; -1 where the warp was skipped); count = pairs * levels * max_warps.
 * Synchronous. */
svs_status svs_tvl1_plan_get_residuals(svs_plan* plan, float* out_host, size_t count);
/* Shape of variant tile_id: tile width and height, prefetch distance, form (0 plain-load, 1 TMA
 * pipeline, 2 split-role TMA pipeline) and voxels per lane (1 or 2); any output may be NULL;
 * SVS_ERR_INVALID_ARG for an unknown id. No counterpart in the reference (a query for the
 * autotuner and tests). */
svs_status svs_tvl1_tile_info(int tile_id, int* tx, int* ty, int* dist, int* form, int* lane_voxels);
/* CTAs of split-role variant tile_id that one SM holds at once for a storage mode (the occupancy
 * calculator on the current device, with the kernel's registers and shared memory); general
 * boundary != 0 for the NEAREST / periodic kernels, 0 for MIRROR. SVS_ERR_UNSUPPORTED for a
 * variant not compiled for the storage or not fitting shared memory. No counterpart in the
 * reference (a query for tests and tuning). */
svs_status svs_tvl1_tile_occupancy(int storage, int tile_id, int general_boundary, int* ctas_per_sm);

/* A plan sized by capacity for svs_tvl1_plan_retarget (no counterpart in the reference): room for
 * up to max_pairs pairs and at least arena_bytes of device state (the per-pair state of a level-0
 * voxel is about 190 bytes with 16-bit fields, 290 with FP32 storage, three scales). It starts
 * with a placeholder batch of max_pairs small cubes; retarget it before solving. */
svs_status svs_tvl1_plan_create_reserve(const svs_tvl1_params* params, int max_pairs, size_t arena_bytes,
                                        svs_plan** plan);
/* Re-use a plan for another batch without allocating (no counterpart in the reference): the plan
 * takes num_pairs pairs with level-0 sizes dims_host[3i..3i+2], num_pairs at most its pair count
 * at creation and their device state at most its arena (SVS_ERR_OUT_OF_MEMORY otherwise); state
 * is cleared on `stream`, tile lists, tensor maps and the solve graph are rebuilt at the next
 * solve, per-pair variant requests are dropped. Not with residuals on. The plan must not be
 * solving on any stream. Used by the serving loop, which packs pairs of several requests into
 * one batch. */
svs_status svs_tvl1_plan_retarget(svs_plan* plan, int num_pairs, const int* dims_host, svs_stream_t stream);

/* Solve every pair of the plan (pairs[i] must match dims[i] of the plan). */
svs_status svs_tvl1_solve_batch(svs_plan* plan, const svs_pair_desc* pairs_host, int num_pairs,
                                svs_stream_t stream);

/* Benchmark hook: launch `count` iterate kernels (the fused primal-dual iteration) of pyramid
 * level `level` on the plan's current state, alternating its ping-pong buffers. Used to time the
 * dominant kernel on live data and by the autotuner; it overwrites the plan's iteration state
 * (results already copied out by svs_tvl1_solve_batch are unaffected). */
svs_status svs_tvl1_bench_iterations(svs_plan* plan, int level, int count, svs_stream_t stream);
/* Number of kernel nodes in the plan's captured solve graph (0 before the first solve). */
uint64_t svs_tvl1_plan_graph_kernels(const svs_plan* plan);
/* Iterate-kernel variant the plan uses at a pyramid level (after the first solve; 0 before). */
int svs_tvl1_plan_level_tile(const svs_plan* plan, int level);
/* Variant one pair runs at a pyramid level: the level's, or its group's (requested with
 * svs_tvl1_plan_set_pair_tile or chosen automatically); after the first solve, 0 before. */
int svs_tvl1_plan_pair_tile_used(const svs_plan* plan, int level, int pair);
/* The automatic variant choice for one pyramid level, host arithmetic only (no counterpart in
 * the reference): num_pairs sizes dims_host[3i..3i+2] = (nz, ny, nx) at that level, storage mode,
 * SM count. Returns the level's variant and writes pair_tile_out[i] = pair i's own variant where
 * it differs (0: the level's); 0 for invalid arguments. 2-byte fields at levels whose 40x8
 * column tiles fill two CTAs per SM at least twice: each pair takes the variant with the least
 * work (column tiles x planes x a measured time per column-tile plane) and the variant with the
 * most work is the level's; otherwise one variant per level (FP32 fields: 32x16 voxel pairs;
 * 2-byte fields: 40x8 voxel pairs when every width is a multiple of 40, 32x8 single voxels up to
 * width 32, 16x16 single voxels otherwise). */
int svs_tvl1_auto_tiles(int storage, int num_pairs, const int* dims_host, int sms, int* pair_tile_out);
/* CTAs of one iteration at a pyramid level, all variant groups together (after the first solve;
 * 0 before): the column tiles times their z chunks. */
int64_t svs_tvl1_plan_level_ctas(const svs_plan* plan, int level);
/* The z-chunk plan of the split-role kernels (host arithmetic only, no device needed): for
 * `columns` column tiles of up to `nz` planes on `slots` resident CTAs (SMs x CTAs per SM), the
 * first columns - tail_columns march in main_chunks chunks each and the last tail_columns in
 * tail_chunks, minimising waves x (planes per chunk + 3) summed over the two phases. */
svs_status svs_tvl1_chunk_plan(int64_t columns, int nz, int64_t slots, int* main_chunks, int* tail_chunks,
                               int64_t* tail_columns);
/* Synchronous check of the plan's device status: SVS_ERR_TIMEOUT if a bounded pipeline wait
 * inside an iterate kernel gave up (the kernel then returned early and the results of the
 * solves since the last check are invalid), SVS_OK otherwise. The status is cleared once it has
 * been reported. */
svs_status svs_tvl1_plan_check(svs_plan* plan);
/* Test hook for the bounded pipeline waits of the TMA iterate kernels (no counterpart in the
 * reference): at pyramid `level`, the CTA with launch index `cta` never issues the copies of its
 * staged plane number `plane` (counted from the first plane it stages), and every pipeline wait
 * gives up after wait_us microseconds (0 = the default, 2 s). The waiting threads then record
 * SVS_DEV_TIMEOUT, the CTA waits (bounded) for the copies it did issue and returns, and
 * svs_tvl1_plan_check reports SVS_ERR_TIMEOUT; the context stays usable. level, cta or plane < 0
 * switches the stall off (wait_us still applies). */
svs_status svs_tvl1_plan_set_stall_test(svs_plan* plan, int level, int cta, int plane, uint32_t wait_us);
/* Persistent iteration loop (no counterpart in the reference, whose tvl13d.py:213-253 launches
 * every operator of every iteration): with on != 0, each warp of a level whose pairs all use one
 * split-role variant that has the persistent form runs its max_outer_iterations iterations in ONE
 * cooperative launch of the resident CTAs, which take the level's column tiles in turn and meet
 * at a grid barrier (bounded wait, SVS_DEV_TIMEOUT on expiry) after every iteration; results are
 * bitwise those of the per-iteration launches. Levels without the form, or a device where the
 * cooperative launch cannot be captured into the solve's graph, keep per-iteration launches. */
svs_status svs_tvl1_plan_set_persistent(svs_plan* plan, int on);
/* 1 if the captured solve graph runs level `level` with the persistent loop, else 0. */
int svs_tvl1_plan_level_persistent(const svs_plan* plan, int level);

/* Allocation-free solve of ONE frame pair, for callers that cannot call cudaMalloc: code whose
 * device memory belongs to another allocator (a framework's caching pool that has reserved the
 * GPU) and latency-critical loops in which an allocation or free would synchronize the device.
 * No counterpart in the reference (its operators allocate every output with torch::zeros).
 * Same result as svs_tvl1_solve_batch with the plain-load iterate kernel (tile id 6) for the
 * same parameters; the caller passes device frames I0, I1 [nz,ny,nx] and the flow u_out
 * [nz,ny,nx,3]. All other device memory the solve needs (pyramid, linearisation, dual state,
 * descriptors, tile lists) is taken from one static 32 MiB device array that every GPU loading
 * the library holds until exit; a volume whose state does not fit is rejected with
 * SVS_ERR_INVALID_ARG. With three scales the largest cubes that fit are 56^3 with FP32 storage
 * (55^3 with the median post-filter), 64^3 with F16/BF16_FLOW32 (63^3 with the median) and
 * 66^3 with F16/BF16 (64^3 with the median). Calls no cudaMalloc or cudaFree; the descriptors
 * and tile lists travel to the device as kernel parameters. The first call on a device (and the
 * first after its context was reset) looks up the array's device address
 * (cudaGetSymbolAddress): make it before any stream capture. Every call reuses the same array
 * and clears the state it uses, so calls that overlap on the GPU (different streams or devices
 * sharing nothing else) race and must be serialized by the caller; the p output and the
 * num_scales == 1 warm start of svs_pair_desc are not offered here. */
svs_status svs_tvl1_solve_noalloc(const svs_tvl1_params* params, const float* I0, const float* I1,
                                  int nz, int ny, int nx, float* u_out, svs_stream_t stream);

/* Kernel-launch counter (all kernels this library launched in this process), for benchmarks. */
uint64_t svs_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* SVSFLOW_H_ */
