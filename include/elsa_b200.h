/*
 * elsa_b200: C ABI of the B200-native X-ray projector + iterative-solver hot path.
 *
 * Plain pointers and sizes only. Device pointers are CUDA device memory of the current device;
 * `stream` is a cudaStream_t (NULL = legacy default stream). Every call returns an elsa_status;
 * on failure elsa_last_error() gives a message (thread-local). No C++ exception crosses this
 * boundary.
 *
 * Data layout (elsa's, core/Descriptors/DataDescriptor.cpp:86-118):
 *   volume   float[nx*ny(*nz)], x fastest
 *   sinogram float[nu(*nv)*num_poses], u fastest, pose last
 *     (core/Descriptors/DetectorDescriptor.cpp:20-52)
 *   pose     40 floats: P (dim x dim+1, row-major) at 0, Pinv (dim+1 x dim) at 12,
 *            camera centre C (dim) at 24, extrinsic ext (dim x dim+1) at 27,
 *            source-detector distance at 39; all in voxel-index units
 *            (core/Geometry.cpp:225-270).
 */
#ifndef ELSA_B200_H
#define ELSA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ELSA_POSE_FLOATS 40

typedef enum elsa_status {
    ELSA_SUCCESS = 0,
    /* dimension mismatch, empty geometry, unsupported dim (elsa: InvalidArgumentError) */
    ELSA_ERROR_INVALID_ARGUMENT = 1,
    /* elsa: LogicError */
    ELSA_ERROR_LOGIC = 2,
    /* device allocation failed (elsa: std::bad_alloc) */
    ELSA_ERROR_BAD_ALLOC = 3,
    /* CUDA runtime error */
    ELSA_ERROR_CUDA = 4,
    /* geometry or option this build does not handle */
    ELSA_ERROR_NOT_SUPPORTED = 5
} elsa_status;

typedef enum elsa_projector_kind {
    /* JosephsMethod / JosephsMethodCUDA, projectors/JosephsMethod.cpp:37-198. params[0] = fast
     * (default 0): 0 = the matched adjoint (the transpose of the forward, as JosephsMethod and
     * JosephsMethodCUDA(..., fast = false)); 1 = JosephsMethodCUDA's `fast` adjoint
     * (JosephsMethodCUDA.h:60-67, TraverseJosephsCUDA.cu:218-287), a voxel-driven backprojection
     * through a texture with linear filtering that is not the transpose (the reference's
     * default; planar detectors only). */
    ELSA_PROJECTOR_JOSEPH = 0,
    /* SiddonsMethod / SiddonsMethodCUDA, projectors/SiddonsMethod.cpp:76-124 with
     * projectors/TraverseAABB.cpp:6-184 */
    ELSA_PROJECTOR_SIDDON = 1,
    /* BlobVoxelProjector / BlobVoxelProjectorCUDA, projectors/VoxelProjector.cpp:7-52.
     * params: radius (2), alpha (10.83), order (2), footprint mode (0). */
    ELSA_PROJECTOR_BLOB = 2,
    /* BSplineVoxelProjector / BSplineVoxelProjectorCUDA, projectors/VoxelProjector.cpp:69-114.
     * params: order (2), footprint mode (0). */
    ELSA_PROJECTOR_BSPLINE = 3,
    /* PhaseContrastBlobVoxelProjector(CUDA), projectors/PhaseContrastProjector.cpp:6-52.
     * params as ELSA_PROJECTOR_BLOB. */
    ELSA_PROJECTOR_PHASE_CONTRAST_BLOB = 4,
    /* PhaseContrastBSplineVoxelProjector(CUDA), projectors/PhaseContrastProjector.cpp:72-119.
     * params as ELSA_PROJECTOR_BSPLINE. */
    ELSA_PROJECTOR_PHASE_CONTRAST_BSPLINE = 5,
    /* BinaryMethod, projectors/BinaryMethod.cpp:66-111: the voxels TraverseAABB visits, each
     * with weight 1 (elsa has it on the CPU only). */
    ELSA_PROJECTOR_BINARY = 6,
    /* BlobProjector, the ray-driven blob projector of projectors/LutProjector.h:85-199 (the
     * slice walk of SliceTraversal.cpp, lut(distance to the ray) for the voxels within
     * ceil(radius) in each slice). params: radius (2), alpha (10.83), order (2). As in the
     * reference, the adjoint walks a box grown by the support, so forward and adjoint are not
     * exact transposes near the volume faces. */
    ELSA_PROJECTOR_RAY_BLOB = 7,
    /* BSplineProjector, the same with the projected B-spline (neighbourhood 2,
     * LutProjector.cpp:48-90). params: order (2). */
    ELSA_PROJECTOR_RAY_BSPLINE = 8
} elsa_projector_kind;

/* Footprint mode of the voxel projectors (last parameter): 0 visits the pixels of each voxel
 * footprint exactly as elsa's CPU loop does (projectors/VoxelComputation.h:88-113, which visits a
 * sheared block when the clamped footprint is not square); 1 visits the footprint rectangle. */
#define ELSA_FOOTPRINT_REFERENCE 0
#define ELSA_FOOTPRINT_RECTANGLE 1

typedef struct elsa_projector elsa_projector;
typedef struct elsa_cgne_split elsa_cgne_split;
typedef struct elsa_batch_cgne elsa_batch_cgne;

/* Message of the last failed call on this thread ("" if none). */
const char* elsa_last_error(void);

/* ABI version of this library. */
int32_t elsa_abi_version(void);

/* ---------------------------------------------------------------------------------------------
 * Geometry
 * ------------------------------------------------------------------------------------------- */

/* One 2D pose. Replaces Geometry(SourceToCenterOfRotation, CenterOfRotationToDetector, Radian,
 * VolumeData2D, SinogramData2D, PrincipalPointOffset, RotationOffset2D),
 * core/Geometry.cpp:12-51. vol_spacing/vol_origin/cor_offset: 2 floats; sino_spacing/
 * sino_origin: 2 floats (only [0] is used). */
elsa_status elsa_pose_2d(float source_to_center, float center_to_detector, float angle_rad,
                         const float* vol_spacing, const float* vol_origin,
                         const float* sino_spacing, const float* sino_origin,
                         float principal_point_offset, const float* cor_offset, float* out_pose);

/* One 3D pose (YZY Euler angles gamma, beta, alpha). Replaces Geometry(..., VolumeData3D,
 * SinogramData3D, RotationAngles3D, PrincipalPointOffset2D, RotationOffset3D),
 * core/Geometry.cpp:53-109. */
elsa_status elsa_pose_3d(float source_to_center, float center_to_detector,
                         const float* vol_spacing, const float* vol_origin,
                         const float* sino_spacing, const float* sino_origin, float gamma,
                         float beta, float alpha, const float* principal_point_offset,
                         const float* cor_offset, float* out_pose);

/* Circular trajectory. Replaces CircleTrajectoryGenerator::createTrajectory,
 * generators/CircleTrajectoryGenerator.cpp:9-24 (with BaseCircleTrajectoryGenerator.cpp:12-74,
 * TrajectoryGenerator.cpp:9-47). det_size (dim-1) and det_spacing (dim-1) may be NULL for
 * elsa's defaults. out_poses: num_poses*ELSA_POSE_FLOATS floats; out_det_dims: dim entries. */
elsa_status elsa_circle_trajectory(int32_t dim, const int64_t* vol_dims, const float* vol_spacing,
                                   int64_t num_poses, float arc_degrees, float source_to_center,
                                   float center_to_detector, const int64_t* det_size,
                                   const float* det_spacing, float* out_poses,
                                   int64_t* out_det_dims);

/* ---------------------------------------------------------------------------------------------
 * Projectors (LinearOperator<float> on device buffers)
 * ------------------------------------------------------------------------------------------- */

/* Create a projector on the current device. vol_dims: dim entries; det_dims: dim entries
 * (nu[, nv], num_poses); poses: host, num_poses*ELSA_POSE_FLOATS floats; params: kind-specific
 * (unused for Joseph, may be NULL). Replaces the constructors JosephsMethodCUDA(VolumeDescriptor,
 * DetectorDescriptor), projectors_cuda/JosephsMethodCUDA.cpp:9-92, and
 * JosephsMethod(VolumeDescriptor, DetectorDescriptor), projectors/JosephsMethod.cpp:11-28. */
elsa_status elsa_projector_create(int32_t kind, int32_t dim, const int64_t* vol_dims,
                                  const int64_t* det_dims, const float* poses,
                                  const float* params, int32_t num_params,
                                  elsa_projector** out);

/* As elsa_projector_create for a curved (cylindrical) detector, CurvedDetectorDescriptor
 * (core/Descriptors/CurvedDetectorDescriptor.cpp:8-120) as CurvedCircleTrajectoryGenerator
 * builds it (generators/CurvedCircleTrajectoryGenerator.cpp:8-30): the same poses, opening
 * angle `angle` (radian, > 0) and source-to-detector distance `s2d` (source-to-centre plus
 * centre-to-detector). The ray of pixel (u, v) passes the pixel centre's point on the arc.
 * Kinds ELSA_PROJECTOR_JOSEPH, _SIDDON and _BINARY; the voxel projectors need a planar
 * detector (ELSA_ERROR_NOT_SUPPORTED). */
elsa_status elsa_projector_create_curved(int32_t kind, int32_t dim, const int64_t* vol_dims,
                                         const int64_t* det_dims, const float* poses,
                                         const float* params, int32_t num_params, float angle,
                                         float s2d, elsa_projector** out);

/* Planar detector coordinates of the pixel centres of a curved detector, two floats (u', v')
 * per pixel, u fastest (v' = 0 in 2D): CurvedDetectorDescriptor::getPlanarCoords. out holds
 * 2 * nu * nv floats (nv = 1 in 2D). Host only. */
elsa_status elsa_curved_detector_coords(int32_t dim, int32_t nu, int32_t nv, float angle,
                                        float s2d, float* out);

/* Replaces the operator's destructor (JosephsMethodCUDA.cpp:94-107). */
elsa_status elsa_projector_destroy(elsa_projector* projector);

/* Domain (volume) and range (sinogram) coefficient counts
 * (LinearOperator::getDomainDescriptor/getRangeDescriptor, core/LinearOperator.h:60-70). */
elsa_status elsa_projector_sizes(const elsa_projector* projector, int64_t* domain_size,
                                 int64_t* range_size);

/* Diagnostics: key 0 = conflict-free ray class spacing of the adjoint, 1 = adjoint bricks,
 * 2 = samples per forward pass (sum over rays of the Joseph step count), 3 = error word of the
 * device pipeline (0 = no timed-out wait; synchronizes), 4 = detector tiles on the gather
 * fallback of the staged forward, in parts per million, 5 = footprint mode of a voxel
 * projector, 6 / 7 = kernel launches per forward / adjoint call, 8 = samples (Joseph taps, Siddon
 * visits) of the brick-owner adjoint that fall outside the window of the brick that owns them
 * (0 = every brick's ray list is complete; runs a check kernel and synchronizes). */
elsa_status elsa_projector_info(const elsa_projector* projector, int32_t key, int64_t* value);

/* Test hook of the bounded device waits (no counterpart in the reference, whose kernels do not
 * wait on one another). The TMA-staged Joseph forward (3D) waits on shared-memory barriers for its
 * volume copies; every wait gives up after a limit (about one second of clock cycles), records
 * bit 0 of the error word (elsa_projector_info key 3), waits (bounded again) for the copies it
 * issued and returns, so the GPU context stays usable. This call sets the limit to waitCycles
 * clock cycles (<= 0: the default) and, with withholdCopies != 0, makes the forward issue no
 * copies, so that every wait runs out: a test of that path without any fault. The forward's
 * output is then undefined. Clears the error word; synchronizes the device. Returns
 * ELSA_ERROR_NOT_SUPPORTED for projectors without bounded waits. */
elsa_status elsa_projector_wait_test(elsa_projector* projector, int64_t waitCycles,
                                     int32_t withholdCopies);

/* Launch parameters ("knobs") of a projector. None of them changes the operator: every value
 * computes the same forward and adjoint up to float rounding (adjoint view chunks only change
 * the order in which per-chunk partial volumes are added). The reference has no counterpart;
 * its CUDA projectors launch fixed block shapes (JosephsMethodCUDA.cpp:132-214,
 * ProjectVoxelsCUDA.cu:21-239). */
#define ELSA_KNOB_FORWARD_THREADS 0 /* rays per block of a thread-per-ray forward (Siddon, 2D Joseph) */
#define ELSA_KNOB_ADJOINT_CHUNKS 1  /* view chunks of a brick-owner adjoint (Joseph, Siddon) */
#define ELSA_KNOB_ADJOINT_THREADS 2 /* voxels per block of a thread-per-voxel adjoint (blob, B-spline) */
/* Adjoint scheme of Joseph (matched adjoint), Siddon and BinaryMethod: 0 = deterministic
 * brick-owner kernel (bit-reproducible), 1 = thread-per-ray atomic scatter, the reference's own
 * scheme (SiddonsMethod.cpp:119 `omp atomic`, TraverseSiddonsCUDA.cu atomicAdd): the same sums
 * in an order that varies from run to run. Default 0 for Joseph; for Siddon / BinaryMethod 0 when
 * the brick owner exists for the geometry (a valid class spacing) and its checkpoint tables
 * (20 bytes per ray and 16-plane slab, about 20 GB at 256^3 / 360 x 384^2) take at most a quarter
 * of the device's memory and half of the free memory at creation, else 1. At 256^3 the Siddon
 * brick owner takes 1.22x the scatter's time. */
#define ELSA_KNOB_ADJOINT_SCATTER 3
/* Weights of the voxel projectors' adjoint (blob, B-spline and their phase-contrast forms):
 * 0 = the forward's weights (distance as n2 * rsqrt(n2), scaling applied as a multiplication by
 * 1 / s, the table lerp as one fma; within a few ulp of the reference's, and forward and adjoint
 * then use the same weights), 1 = the reference's float operations (VoxelComputation.h:55-185),
 * the adjoint bit-identical to elsa's CPU loop. Default 0 (1.4x faster). Either way the adjoint
 * is deterministic. */
#define ELSA_KNOB_EXACT_WEIGHTS 4
/* Planes per checkpoint slab of the 3D Joseph matched adjoint: 16, 32, 64 or 128. The adjoint
 * replays every ray from its exact accumulated position at the slab's first sample (8 bytes per
 * ray and slab); deeper slabs need less memory and add catch-up additions to bricks inside a
 * slab, with the same results bit for bit. Default: the smallest depth whose table takes at most
 * an eighth of the device's memory (16 at 256^3 / 360 x 384^2, 8.1 GB). Setting it rebuilds the
 * table (synchronizes the device). */
#define ELSA_KNOB_CHECKPOINT_DEPTH 5
#define ELSA_KNOB_COUNT 6

/* Current value of `knob` (-1: the projector does not use it). */
elsa_status elsa_projector_get_knob(const elsa_projector* projector, int32_t knob,
                                    int32_t* value);

/* Candidate values of `knob` for this projector's geometry, ascending: *count receives their
 * number (0: not tunable here) and the first min(*count, capacity) are written to values. */
elsa_status elsa_projector_knob_candidates(const elsa_projector* projector, int32_t knob,
                                           int32_t* values, int32_t capacity, int32_t* count);

/* Set `knob` to one of its candidates (or, for the adjoint chunks, the default the projector
 * chose at creation); other values return ELSA_ERROR_INVALID_ARGUMENT. May allocate or free the
 * adjoint's partial volumes; synchronous with respect to the host. */
elsa_status elsa_projector_set_knob(elsa_projector* projector, int32_t knob, int32_t value);

/* Autotuner: time every candidate of every knob (the forward for the forward knob, the adjoint
 * for the others) with CUDA events on `stream`, keep the fastest, and record the choice in the
 * process-wide tuning cache under the key "kind:dim:nx,ny,nz:nu,nv,np". Unless `force` is
 * non-zero, a key already in the cache is applied without timing. values (may be NULL) receives
 * ELSA_KNOB_COUNT values (-1 for unused knobs); *from_cache (may be NULL) is set to 1 when the
 * cache supplied them. Allocates one volume and one sinogram of scratch; synchronizes `stream`.
 * No reference counterpart. */
elsa_status elsa_projector_autotune(elsa_projector* projector, void* stream, int32_t force,
                                    int32_t* values, int32_t* from_cache);

/* The tuning cache (host memory, shared by all threads): number of entries, removal of all
 * entries, writing it to a text file (one line per key: the key and ELSA_KNOB_COUNT integers)
 * and reading such a file (adding to or replacing the entries; a malformed file changes
 * nothing and returns ELSA_ERROR_INVALID_ARGUMENT). Set and look up one entry directly with
 * elsa_tune_cache_put / elsa_tune_cache_get (*found = 0 when absent). No reference counterpart. */
elsa_status elsa_tune_cache_size(int64_t* entries);
elsa_status elsa_tune_cache_clear(void);
elsa_status elsa_tune_cache_save(const char* path);
elsa_status elsa_tune_cache_load(const char* path);
elsa_status elsa_tune_cache_put(const char* key, const int32_t* values);
elsa_status elsa_tune_cache_get(const char* key, int32_t* values, int32_t* found);

/* y = A x on device buffers. Replaces LinearOperator::apply(x, Ax), core/LinearOperator.cpp:94-98
 * -> XrayProjector::applyImpl -> JosephsMethodCUDA::forward, JosephsMethodCUDA.cpp:132-214.
 * Asynchronous on `stream`.
 * Concurrency: a projector owns device scratch that its applies write (the TMA forward's
 * permuted copies of x, the adjoint's per-view-chunk partial volumes, staging buffers of the
 * host-buffer entry points). Applies of ONE projector must therefore be ordered: issue them on
 * one stream, or order the streams with events. Different projectors (also of the same geometry)
 * may run concurrently on any streams. The reference's CUDA projectors are not reentrant either
 * (they share the device and synchronize it on every call). */
elsa_status elsa_projector_apply(elsa_projector* projector, const float* x, float* y,
                                 void* stream);

/* x = A^T y on device buffers (matched, atomic-free, deterministic). Replaces
 * LinearOperator::applyAdjoint(y, Aty), core/LinearOperator.cpp:182-186 ->
 * JosephsMethodCUDA::backward, JosephsMethodCUDA.cpp:216-389. */
elsa_status elsa_projector_apply_adjoint(elsa_projector* projector, const float* y, float* x,
                                         void* stream);

/* Batched applies on device buffers: for b < batch, y + b yStride = A (x + b xStride)
 * (elsa_projector_apply_batch) or x + b xStride = A^T (y + b yStride)
 * (elsa_projector_apply_adjoint_batch); strides in floats, at least the element sizes. Each
 * element equals what the single-volume entry point computes, bit for bit. The 3D Joseph
 * operator runs the whole batch in one launch per kernel, sharing its ray tables; the other
 * operators apply the elements in turn. No reference counterpart: elsa applies one DataContainer
 * at a time (LinearOperator::apply, core/LinearOperator.cpp:94-98); this serves batched
 * (differentiable) reconstruction. Same concurrency rule as the single applies. */
elsa_status elsa_projector_apply_batch(elsa_projector* projector, const float* x,
                                       int64_t xStride, float* y, int64_t yStride, int32_t batch,
                                       void* stream);
elsa_status elsa_projector_apply_adjoint_batch(elsa_projector* projector, const float* y,
                                               int64_t yStride, float* x, int64_t xStride,
                                               int32_t batch, void* stream);

/* Host-buffer variants, synchronous: copy the input to the device, run, copy the output back
 * (the call pattern of the reference's CUDA projectors, which copy in and out on every apply,
 * JosephsMethodCUDA.cpp:132-214). For the 3D Joseph operator (matched adjoint in view chunks)
 * the copies of the sinogram overlap the kernels: the forward copies finished groups of views
 * out while later groups run, the adjoint copies groups of views in while earlier groups run
 * (page-locked host buffers let the copies run asynchronously). Results equal the device-buffer
 * entry points bit for bit. */
elsa_status elsa_projector_apply_host(elsa_projector* projector, const float* x, float* y);
elsa_status elsa_projector_apply_adjoint_host(elsa_projector* projector, const float* y,
                                              float* x);

/* ---------------------------------------------------------------------------------------------
 * Vector operations on device float buffers; scalar results are float64 in device memory
 * ------------------------------------------------------------------------------------------- */

/* *result = <x, y>, accumulated in float64 in a fixed order (bit-reproducible). Replaces
 * DataContainer::dot, core/DataContainer.cpp:403-417 (storage/reductions/DotProduct.h:24-47).
 * result is device memory; the call is asynchronous on `stream` (read the result after the
 * stream's work). Its partial sums come from the device's stream-ordered memory pool
 * (cudaMallocAsync / cudaFreeAsync on `stream`), which neither synchronizes the device nor waits
 * on the host. */
elsa_status elsa_dot(const float* x, const float* y, int64_t n, double* result, void* stream);

/* Largest n accepted by elsa_dot_no_alloc. */
#define ELSA_DOT_NO_ALLOC_MAX_ELEMENTS ((int64_t)67108864)

/* *result = <x, y> like elsa_dot, but without allocating any device memory. No counterpart in
 * the reference: it exists for callers that must not call cudaMalloc/cudaFree (those synchronize
 * the whole device and stall other streams, and some hosts route all device memory through their
 * own pool). The partial sums live in a fixed 128 KiB device array that the library keeps on
 * every GPU that loads it, so n is limited to ELSA_DOT_NO_ALLOC_MAX_ELEMENTS (larger n returns
 * ELSA_ERROR_INVALID_ARGUMENT). result is device memory; the call is asynchronous on `stream`.
 * All calls on a device share the array: calls that may run at the same time on the GPU race and
 * must be ordered on one stream. The first call on a device looks up the array's device address;
 * make that first call before any stream capture. The address is kept for the life of the
 * process, so a device reset (cudaDeviceReset) after that first call is not supported. */
elsa_status elsa_dot_no_alloc(const float* x, const float* y, int64_t n, double* result,
                              void* stream);

/* *result = |x|_2^2, like elsa_dot (float64, asynchronous, result in device memory). Replaces
 * DataContainer::squaredL2Norm (storage/reductions/L2.h:15-49). */
elsa_status elsa_squared_l2_norm(const float* x, int64_t n, double* result, void* stream);

/* out = a*x + b*y. Replaces lincomb(a, x, b, y, out), core/DataContainer.cpp:1075-1108
 * (storage/transforms/Lincomb.h:28-33). */
elsa_status elsa_lincomb(float a, const float* x, float b, const float* y, float* out, int64_t n,
                         void* stream);

/* Lookup table (100 samples on [0, support]) that a voxel projector kind uses for dimension dim:
 * the projected blob / B-spline, its derivative (2D phase contrast) or its derivative / s (3D
 * phase contrast). params as for elsa_projector_create. Replaces ProjectedBlob::get_lut,
 * get_derivative_lut, get_normalized_gradient_lut (projectors/Blobs.h:233-300) and the
 * ProjectedBSpline ones (projectors/BSplines.h:132-200). out: host array of `samples` floats. */
elsa_status elsa_voxel_lut(int32_t kind, int32_t dim, const float* params, int32_t num_params,
                           int32_t samples, float* out, float* support);

/* ---------------------------------------------------------------------------------------------
 * Solvers (device-resident iterations, float64 inner products)
 * ------------------------------------------------------------------------------------------- */

typedef struct elsa_solver elsa_solver;

typedef enum elsa_solver_kind {
    /* CGNE<float>, solvers/CGNE.cpp:20-78. params: none. */
    ELSA_SOLVER_CGNE = 0,
    /* CGLS<float>, solvers/CGLS.cpp:12-91. params[0] = eps (damping eps^2, default 0),
     * params[1] = tol (stop once |A^T s - eps^2 x|^2 < tol, default 1e-4). */
    ELSA_SOLVER_CGLS = 1,
    /* Landweber<float>, solvers/LandweberIteration.cpp:26-72 + Landweber.cpp:20-25.
     * params[0] = step size (<= 0 or absent: 0.9 * 2 / powerIterations(A^T A)). */
    ELSA_SOLVER_LANDWEBER = 2,
    /* APGD<float> (FISTA), solvers/APGD.cpp:14-102. params[0] = mu (<= 0 or absent:
     * 0.45 / powerIterations(A^T A)), params[1] = epsilon (stop once |grad|^2 <= epsilon, default
     * FLT_EPSILON), params[2] = proximal operator: 0 identity, 1 box constraint
     * (proximal_operators/ProximalBoxConstraint.cpp:20-40), 2 L1
     * (proximal_operators/ProximalL1.cpp:21-33); params[3] = lower bound, params[4] = upper
     * bound (NaN = no bound; box only), params[5] = L1 weight sigma (default 1). */
    ELSA_SOLVER_APGD = 3,
    /* SIRT<float>, solvers/SIRT.cpp:8-45 (Landweber with T A^T M, M = 1/(A 1 + 1e-10),
     * T = 1/(A^T 1)). params[0] = step size (<= 0 or absent: 0.9 * 2 / powerIterations(T A^T M A)).
     */
    ELSA_SOLVER_SIRT = 4,
    /* FGM<float> on LeastSquares(A, b), solvers/FGM.cpp:33-78. params[0] = epsilon (stop once
     * |grad|^2 <= epsilon^2 |grad_0|^2, default FLT_EPSILON). */
    ELSA_SOLVER_FGM = 5,
    /* OGM<float> on LeastSquares(A, b), solvers/OGM.cpp:40-95 (20 power iterations for the
     * Lipschitz constant). params[0] = epsilon as FGM. The last iteration of each
     * elsa_solver_iterate call uses OGM's final-step factor, so one call of n iterations matches
     * OGM::solve(n). */
    ELSA_SOLVER_OGM = 6,
    /* SQS<float> on LeastSquares(A, b) without subsets, solvers/SQS.cpp:87-170 (diagonal
     * majorizer 1 / (A^T A 1)). params[0] = momentum acceleration (1 default, 0 off),
     * params[1] = epsilon (stop once |grad|^2 <= epsilon^2 |grad_0|^2, default FLT_EPSILON).
     * Ordered subsets and a preconditioner: elsa_sqs_create. */
    ELSA_SOLVER_SQS = 7
} elsa_solver_kind;

/* Many CGNE solves advanced together (a batch of reconstructions of uneven size; no reference
 * counterpart: elsa solves one problem at a time, CGNE.cpp:20-78 per DataContainer). Instance i
 * solves A_i^T A_i x_i = A_i^T b_i from x_i = 0 with its own operator (a 3D Joseph projector
 * with the matched adjoint; others return ELSA_ERROR_NOT_SUPPORTED), b_i and x_i device
 * buffers. Per iteration the instances' forwards run concurrently, all adjoints run in one
 * launch per driving-axis grid over an instance table, and all vector updates in five launches;
 * every x_i equals what a single elsa_solver session computes, bit for bit.
 * elsa_batch_cgne_iterate_graph captures the batched iterations as one CUDA graph (stream must
 * be an explicitly created stream). residuals: count doubles |r_i|^2 in host memory
 * (synchronizes). The projectors must outlive the batch; each belongs to one batch at a time. */
elsa_status elsa_batch_cgne_create(elsa_projector* const* projectors, const float* const* b,
                                   float* const* x, int32_t count, void* stream,
                                   elsa_batch_cgne** out);
elsa_status elsa_batch_cgne_iterate(elsa_batch_cgne* batch, int32_t iterations, void* stream);
elsa_status elsa_batch_cgne_iterate_graph(elsa_batch_cgne* batch, int32_t iterations,
                                          void* stream);
elsa_status elsa_batch_cgne_residuals(elsa_batch_cgne* batch, double* residuals, void* stream);
elsa_status elsa_batch_cgne_destroy(elsa_batch_cgne* batch);

/* CGNE split around the reduction of its normal-operator results (view-sharded solves over
 * several GPUs, one process each; no reference counterpart: multi-GPU solves are a stated goal
 * of elsa's roadmap, ROADMAP.md:48-50). With A = [A_0; A_1; ...] by blocks of views,
 * A^T A = sum_r A_r^T A_r: every rank holds the whole volume and its block's projector
 * (created on its poses), computes its local volumes into caller buffers, the caller sums them
 * across the ranks in place (e.g. an NCCL all-reduce on the same stream), and every rank then
 * performs the same update, so all ranks hold identical x and scalars. Per solve:
 *   elsa_cgne_split_backproject(c, b_r, atb)  atb = A_r^T b_r;   all-reduce atb
 *   elsa_cgne_split_begin(c, atb)             x = 0, r = d = atb, |r|^2
 * per iteration:
 *   elsa_cgne_split_normal(c, q)              q = A_r^T A_r d;   all-reduce q
 *   elsa_cgne_split_update(c, q)              alpha, x, r, beta, d (solvers/CGNE.cpp:50-73)
 * Scalars stay in device memory and no call waits on the host. elsa_cgne_split_residual copies
 * the current |r|^2 (float64) to device memory `result`. x is the caller's volume buffer. */
elsa_status elsa_cgne_split_create(elsa_projector* projector, float* x, elsa_cgne_split** out);
elsa_status elsa_cgne_split_backproject(elsa_cgne_split* cgne, const float* b, float* atb,
                                        void* stream);
elsa_status elsa_cgne_split_begin(elsa_cgne_split* cgne, const float* atb, void* stream);
elsa_status elsa_cgne_split_normal(elsa_cgne_split* cgne, float* q, void* stream);
elsa_status elsa_cgne_split_update(elsa_cgne_split* cgne, const float* q, void* stream);
elsa_status elsa_cgne_split_residual(const elsa_cgne_split* cgne, double* result, void* stream);
elsa_status elsa_cgne_split_destroy(elsa_cgne_split* cgne);

/* Set up a solver run: allocate its scratch, compute the initial residual (x is zeroed unless
 * use_x0 != 0). b (range) and x (domain) are device buffers that must stay valid until
 * elsa_solver_destroy; x holds the current iterate. params (num_params doubles, may be NULL when
 * num_params == 0) are the solver's constructor arguments, laid out per kind as above; missing
 * trailing entries take the reference's defaults. The constructor + first half of
 * Solver::solve(iterations, x0), solvers/Solver.h:21-43. Step sizes derived by power iterations
 * synchronize the stream once. */
elsa_status elsa_solver_create(int32_t kind, elsa_projector* projector, const float* b, float* x,
                               int32_t use_x0, const double* params, int32_t num_params,
                               void* stream, elsa_solver** out);

/* SQS with ordered subsets, solvers/SQS.cpp:10-22,87-170: the constructor
 * SQS(problem, subsets, [preconditioner,] momentumAcceleration, epsilon) + the first half of
 * solve(). projector / b: the full problem LeastSquares(A, b) (device buffer b); subset i:
 * LeastSquares(subset_projectors[i], subset_b[i]) with subset_b[i] that subset's measurements
 * (device buffers, e.g. from elsa_gather_views), every subset projector sharing the volume and
 * having at most the full problem's views; num_subsets 0 solves the full problem, otherwise it
 * must be >= 2. preconditioner: NULL or a device volume buffer p, the diagonal operator applied
 * to every gradient (a Scaling preconditioner). With subsets, each subset step whose gradient
 * passes the threshold is confirmed with the full gradient on the host (one stream
 * synchronization per subset step), so such a solver cannot run as a CUDA graph
 * (elsa_solver_iterate_graph / elsa_solve_batch return ELSA_ERROR_NOT_SUPPORTED). The
 * projectors and buffers must outlive the solver. */
elsa_status elsa_sqs_create(elsa_projector* projector, const float* b,
                            elsa_projector* const* subset_projectors, const float* const* subset_b,
                            int32_t num_subsets, float* x, int32_t use_x0, int32_t momentum,
                            double epsilon, const float* preconditioner, void* stream,
                            elsa_solver** out);

/* Ordered-subset sampling strategies, projectors/SubsetSampler.h:28-31. */
#define ELSA_SUBSET_ROUND_ROBIN 0
#define ELSA_SUBSET_ROTATIONAL_CLUSTERING 1

/* Split num_poses poses (pose records as elsa_projector_create takes them) into num_subsets >= 2
 * subsets (SubsetSampler::splitRoundRobin / splitRotationalClustering,
 * projectors/SubsetSampler.cpp:50-103). view_order (num_poses entries) receives the pose indices
 * subset by subset, subset_sizes (num_subsets entries) the number of poses per subset. Host
 * only. */
elsa_status elsa_subset_split(int32_t dim, const float* poses, int32_t num_poses,
                              int32_t num_subsets, int32_t strategy, int32_t* view_order,
                              int32_t* subset_sizes);

/* out[j] = sinogram view view_order[j] (view_size floats each; device buffers, host index array;
 * asynchronous on `stream`): the per-subset measurement blocks of
 * SubsetSampler::getPartitionedData, projectors/SubsetSampler.cpp:120-150. */
elsa_status elsa_gather_views(const float* sinogram, int64_t view_size, const int32_t* view_order,
                              int32_t num_views, int32_t total_views, float* out, void* stream);

/* Step size in use (Landweber / SIRT step, APGD mu, FGM / OGM 1 / Lipschitz; 0 for the CG
 * solvers and SQS). */
elsa_status elsa_solver_step_size(elsa_solver* solver, double* value);

/* Largest eigenvalue of A^T A by `iterations` power iterations from u = 1, in float with float64
 * inner products. Replaces powerIterations(adjoint(A) * A, iterations),
 * solvers/PowerIterations.cpp:10-27. Synchronizes the stream. */
elsa_status elsa_power_iterations(elsa_projector* projector, int32_t iterations, void* stream,
                                  double* value);

/* Enqueue `iterations` iterations on the stream without synchronizing (the loop bodies of
 * CGNE.cpp:50-73, CGLS.cpp:53-83, LandweberIteration.cpp:57-67, APGD.cpp:64-92). All scalars
 * stay in device memory (a convergence test sets a device flag after which iterations leave the
 * iterate unchanged), so the enqueued work can be captured in a CUDA graph when timing is
 * disabled. */
elsa_status elsa_solver_iterate(elsa_solver* solver, int32_t iterations, void* stream);

/* Like elsa_solver_iterate, but the iterations run as one CUDA graph: captured on the first call
 * (and again whenever `iterations` changes), launched on every call. `stream` must be a created
 * stream (not the legacy default stream) and timing must be off. */
elsa_status elsa_solver_iterate_graph(elsa_solver* solver, int32_t iterations, void* stream);

/* Batched solves: `iterations` iterations of each of the n solvers (distinct projectors and
 * buffers), each as its CUDA graph, spread round-robin over `num_streams` concurrent streams (1 to
 * 64); returns when all have finished. Replaces a loop of Solver::solve calls over independent
 * problems (no reference counterpart for the concurrency). */
elsa_status elsa_solve_batch(elsa_solver* const* solvers, int32_t n, int32_t iterations,
                             int32_t num_streams);

/* Squared norm used by the solver's convergence test (CGNE/CGLS: |r|^2 of the current iterate;
 * APGD: |grad|^2 of the last iteration; Landweber: 0). float64, synchronizes the stream. */
elsa_status elsa_solver_squared_residual(elsa_solver* solver, void* stream, double* value);

/* Record CUDA events around the forward and adjoint projections of every iteration
 * (elsa's Timer around each apply, logging/Timer.h:25-38). */
elsa_status elsa_solver_enable_timing(elsa_solver* solver, int32_t enable);

/* Synchronize and return the total forward / adjoint milliseconds and the number of timed
 * iterations since timing was enabled. */
elsa_status elsa_solver_timing(elsa_solver* solver, double* forward_ms, double* adjoint_ms,
                               int64_t* iterations);

elsa_status elsa_solver_destroy(elsa_solver* solver);

/* CG on the normal equations A^T A x = A^T b. x: device volume buffer, used as the start value
 * when use_x0 != 0 and overwritten with the solution. Replaces CGNE<float>(A, b).solve(
 * iterations, x0), solvers/CGNE.cpp:20-78. */
elsa_status elsa_cgne_solve(elsa_projector* projector, const float* b, float* x,
                            int32_t iterations, int32_t use_x0, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Image files (io/EDFHandler, io/MHDHandler, io/PGMHandler). Host buffers of float; a caller
 * copies them to or from device buffers. Headers are written byte for byte as the reference
 * writes them; reading follows the reference's parse rules and rejects what it rejects
 * (ELSA_ERROR_INVALID_ARGUMENT with the reference's message).
 * ------------------------------------------------------------------------------------------- */

#define ELSA_IO_MAX_DIMS 8

/* Element types of the raw data, DataUtils::DataType (io/ioUtils.h:33-45). Readable: uint16,
 * float32, float64 (converted to float); written: float32. */
#define ELSA_IO_INT8 0
#define ELSA_IO_UINT8 1
#define ELSA_IO_INT16 2
#define ELSA_IO_UINT16 3
#define ELSA_IO_INT32 4
#define ELSA_IO_UINT32 5
#define ELSA_IO_FLOAT32 6
#define ELSA_IO_FLOAT64 7

typedef struct elsa_image_info {
    int32_t ndim;      /* number of dimensions (<= ELSA_IO_MAX_DIMS) */
    int32_t data_type; /* ELSA_IO_* of the stored data */
    int64_t dims[ELSA_IO_MAX_DIMS];   /* coefficients per dimension, x first */
    float spacing[ELSA_IO_MAX_DIMS];  /* spacing per dimension (1 when the file has none) */
} elsa_image_info;

/* Header of an EDF file (EDF::readHeader + parseHeader, io/EDFHandler.cpp:71-216). */
elsa_status elsa_edf_info(const char* path, elsa_image_info* info);
/* Its data, count = the product of the dimensions, converted to float (EDF::read,
 * io/EDFHandler.cpp:9-41). */
elsa_status elsa_edf_read(const char* path, float* out, int64_t count);
/* EDF::write (io/EDFHandler.cpp:43-69,218-255) of float data; spacing may be NULL (ones). */
elsa_status elsa_edf_write(const char* path, const float* data, int32_t ndim, const int64_t* dims,
                           const float* spacing);

/* MHD meta file + raw file (io/MHDHandler.cpp:9-66,68-194); the raw file named in the meta
 * file is found relative to the meta file's directory. */
elsa_status elsa_mhd_info(const char* meta_path, elsa_image_info* info);
elsa_status elsa_mhd_read(const char* meta_path, float* out, int64_t count);
elsa_status elsa_mhd_write(const char* meta_path, const char* raw_path, const float* data,
                           int32_t ndim, const int64_t* dims, const float* spacing);

/* PGM::write (io/PGMHandler.cpp:20-58): 2D data (or 3D with a last dimension of 1) as a P2
 * grey-scale image scaled to [0, 255]. */
elsa_status elsa_pgm_write(const char* path, const float* data, int32_t ndim,
                           const int64_t* dims);

#ifdef __cplusplus
}
#endif

#endif /* ELSA_B200_H */
