/*
 * partia_b200.h -- C ABI of the B200-native SPH interpolation hot path.
 *
 * This is the drop-in boundary for Partia.jl's GPU backend.  Partia selects a
 * backend by Julia multiple dispatch on a singleton type
 * (src/julia/KernelInterpolation/ExecutionBackend/AbstractExecutionBackend.jl:1-2,
 * src/julia/ExtDummy/CUDAExtDummy.jlh:12); the CUDA extension adds methods of
 * `Partia.PointSamples_interpolation` and `Partia.LineSamples_interpolation`
 * (ext/CUDAExt/KernelInterpolation/grid_interpolation/drivers/PointSamples_driver.jl:12,44,
 *  ext/CUDAExt/KernelInterpolation/grid_interpolation/drivers/LineSamples_driver.jl:11,49).
 * A B200 backend implements the same methods by `ccall`ing the functions below.
 *
 * Conventions
 *  - Every function returns PSB_OK (0) or a negative psb_status.  No C++
 *    exception and no longjmp crosses this boundary.  psb_last_error() gives a
 *    one-line message for the last failing call on that context.
 *  - Plain pointers and sizes only.  Unless PSB_FLAG_DEVICE_PTRS is passed,
 *    sample, smoothing-length and output pointers are caller-owned HOST
 *    buffers; the library copies them to and from the device inside the call.
 *    With PSB_FLAG_DEVICE_PTRS they are device pointers on the context's device
 *    and no host<->device copy happens.  Each is checked on the host before
 *    any work is queued: pageable host memory or another device's memory is
 *    refused with PSB_EINVAL (managed memory and page-locked host memory
 *    mapped at the same address are accepted).  Buffer lengths cannot be
 *    checked this way and remain the caller's contract.
 *  - Element type of particle, sample and output arrays is the context dtype
 *    chosen in psb_set_particles (double for PSB_F64, float for PSB_F32),
 *    matching Partia's single float type TF per InterpolationInput.
 *  - Indices exchanged through psb_get_tree use the reference's unified
 *    1-based node ids (internal 1..n-1, leaves n..2n-1, 0 = none)
 *    (src/julia/LinearBoundingVolumeHierarchy/BinaryRadixTree/BinaryRadixTree.jl:37-43).
 *    Permutations and column slots are 0-based.
 *  - A context owns one CUDA stream and its device buffers (particles in
 *    Morton order, the LBVH, reusable scratch).  Calls are synchronous with
 *    respect to the caller.  A context is not thread-safe: use one per host
 *    thread.
 *  - Each call makes the context's device current while it runs and restores
 *    the caller's current device before it returns.
 */
#ifndef PARTIA_B200_H
#define PARTIA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSB_ABI_VERSION 1

typedef struct psb_ctx psb_ctx;

typedef enum {
    PSB_OK = 0,
    PSB_EINVAL = -1,       /* invalid argument (ArgumentError in Partia)            */
    PSB_EDIM = -2,         /* length mismatch (DimensionMismatch in Partia)         */
    PSB_ENOMEM = -3,       /* device or host allocation failed                      */
    PSB_ECUDA = -4,        /* a CUDA runtime call failed                            */
    PSB_ETRAVERSAL = -5,   /* a device loop hit its iteration bound (corrupt tree)  */
    PSB_EUNSUPPORTED = -6, /* option not provided by this build                     */
    PSB_ESTATE = -7        /* call order violated (e.g. interpolate before build)   */
} psb_status;

typedef enum { PSB_F64 = 0, PSB_F32 = 1 } psb_dtype;

/* SPH kernel families of src/julia/KernelInterpolation/kernel_function/kernels/ (one file each):
 * support K h (KernelFunctionValid: 2, 2.5, 3, 2, 2, 2), the 3D norm and f, f'
 * of each file, and each family's line-integrated table
 * (table/line_integrated_kernel_tables.jl).  The adjoint calls differentiate
 * whichever of them the particles were set with. */
typedef enum {
    PSB_KERNEL_M4 = 0,
    PSB_KERNEL_M5 = 1,
    PSB_KERNEL_M6 = 2,
    PSB_KERNEL_C2 = 3,
    PSB_KERNEL_C4 = 4,
    PSB_KERNEL_C6 = 5
} psb_kernel;

/* itpGather / itpScatter / itpSymmetric
 * (src/julia/KernelInterpolation/interpolation_setup/InterpolationStrategy.jl:3-5). */
typedef enum { PSB_GATHER = 0, PSB_SCATTER = 1, PSB_SYMMETRIC = 2 } psb_strategy;

/* Arithmetic of the kernel-weighted sums.  PSB_PREC_FP64: all in double.
 * PSB_PREC_FP32C: pair sums in float with compensated (two-sum) accumulation;
 * for double inputs the neighbour inclusion test and the finalisation
 * (Shepard ratio, A~ subtraction) stay in double, so neighbour sets are the
 * same as in PSB_PREC_FP64. */
typedef enum { PSB_PREC_FP64 = 0, PSB_PREC_FP32C = 1 } psb_precision;

/* Where the sample smoothing length h_a (gather / symmetric) comes from.
 * PSB_H_NEAREST: h of the nearest particle, as Partia's point driver does
 *   (src/julia/KernelInterpolation/grid_interpolation/kernels/PointSamples_kernel.jl:19,
 *    src/julia/LinearBoundingVolumeHierarchy/LinearBVH/LinearBVHQueries.jl:118-140).
 * PSB_H_PER_SAMPLE: hs[i] per sample.   PSB_H_CONSTANT: hs[0] for all samples. */
typedef enum { PSB_H_NEAREST = 0, PSB_H_PER_SAMPLE = 1, PSB_H_CONSTANT = 2 } psb_hmode;

/* Bit flags of the interpolation calls. */
#define PSB_FLAG_DEVICE_PTRS 1u  /* sample / hs / output pointers are device pointers */
/* psb_neighbor_digest only: take the accept/reject decisions of the
 * PSB_PREC_FP32C path (float tests with double fallback) instead of the
 * double ones.  Both must give identical digests. */
#define PSB_FLAG_FP32C_DECISIONS 0x100u
/* Point interpolation normally runs as two kernels (pair
 * lists, then pair sums).  This flag runs the single-kernel form instead, for
 * comparisons; results agree to rounding. */
#define PSB_FLAG_SINGLE_KERNEL 0x200u
/* Line-integrated samples: use a 1000-entry float table of the M4 line
 * integral (the tabulation the benchmark configuration names) instead of the
 * 4096-entry table of the reference (table/line_integrated_kernel_tables.jl:1,
 * looked up as in kernel_function/line_integrated_kernel.jl:13-19).  Both
 * come from the same quadrature; the short table adds its interpolation and
 * float rounding error.  No effect on point samples or the adjoint. */
#define PSB_FLAG_LUT1000_F32 0x400u
/* Point samples: the density gradient (catalog grad slot -1) in the form of
 * the standalone _gradient_density_kernel
 * (src/julia/KernelInterpolation/single_point_interpolation/kernels/gradient_interpolation.jl:1-170):
 * grad rho = sum m gradW - rho(r) sum (m/rho_b) gradW with the plain density
 * sum rho(r) = sum m W, NaN where rho(r) = 0; without the flag the catalog
 * form of general_interpolation.jl:147-169 subtracts the Shepard-normalised
 * density (sum m W) / S1 instead.  Also honoured by the adjoint calls. */
#define PSB_FLAG_DENSITY_GRADIENT_PLAIN 0x800u
/* psb_density only: the number density sum_b W (every mass taken as 1) of
 * _number_density_kernel
 * (src/julia/KernelInterpolation/single_point_interpolation/kernels/scalar_interpolation.jl:86-166),
 * 0 where there is no neighbour. */
#define PSB_FLAG_NUMBER_DENSITY 0x1000u

/* InterpolationCatalogConcise
 * (src/julia/KernelInterpolation/interpolation_setup/InterpolationCatalog.jl:26-32),
 * with 0-based column slots.  A gradient slot of -1 selects the gradient of the
 * particle density itself (the reference's grad slot 0,
 * single_point_interpolation/kernels/general_interpolation.jl:76-82).
 * Outputs are written in the catalog order of
 * grid_interpolation/kernels/PointSamples_kernel.jl:30-71: scalars, then 3 per
 * gradient, then 1 per divergence, then 3 per curl. */
typedef struct {
    int32_t n_scalar;
    const int32_t* scalar_slots;   /* n_scalar                                    */
    const uint8_t* scalar_shepard; /* n_scalar; 1 = Shepard-normalise              */
    int32_t n_grad;
    const int32_t* grad_slots;     /* n_grad                                      */
    int32_t n_div;
    const int32_t* div_slots;      /* 3 * n_div  (x, y, z component columns)      */
    int32_t n_curl;
    const int32_t* curl_slots;     /* 3 * n_curl                                  */
} psb_catalog;

/* Optional per-call statistics; device times are CUDA-event times on the
 * context stream. */
typedef struct {
    double total_ms;       /* whole call, first to last event                    */
    double h2d_ms;         /* host -> device copies inside the call              */
    double order_ms;       /* sample Morton ordering                             */
    double nearest_ms;     /* nearest-particle h pass                            */
    double interp_ms;      /* traversal + kernel-weighted sums                   */
    double d2h_ms;         /* device -> host copies inside the call              */
    int64_t pairs;         /* accepted (sample, particle) pairs                  */
    int64_t exact_retests; /* FP32C pairs re-decided in double near the support  */
    int64_t warp_steps;    /* tree-walk steps summed over warps                  */
    int64_t spans;         /* leaf spans processed (summed over warps)           */
    int64_t span_tests;    /* (span, sample) pairs tested                        */
    int64_t body_iters;    /* pair-body loop iterations summed over warps        */
    int32_t launches;      /* kernels launched by the call                       */
    int32_t reserved;
} psb_stats;

/* ---- context -------------------------------------------------------------- */
int32_t psb_abi_version(void);
int psb_create(psb_ctx** ctx, int device);
int psb_destroy(psb_ctx* ctx);
const char* psb_last_error(const psb_ctx* ctx);
/* Use the caller's CUDA stream (a cudaStream_t) instead of the context's own;
 * NULL restores the context stream. */
int psb_set_stream(psb_ctx* ctx, void* stream);

/* ---- particles and LBVH build -------------------------------------------- */

/* InterpolationInput (src/julia/KernelInterpolation/interpolation_setup/InterpolationInput.jl:41-49,83-107):
 * n particles, coordinates, mass, smoothing length, density and ncol extra
 * columns, all of element type dt.  Pointers are host pointers unless
 * PSB_FLAG_DEVICE_PTRS is set.  The data are copied; the caller's arrays are
 * not modified.  Invalidates any previous LBVH.  kernel is the input's
 * smoothed_kernel (InterpolationInput.jl:49); it sets the support radius of
 * every later query and the kernel evaluated in the sums. */
int psb_set_particles(psb_ctx* ctx, int64_t n, psb_dtype dt,
                      const void* x, const void* y, const void* z,
                      const void* m, const void* h, const void* rho,
                      int32_t ncol, const void* const* cols,
                      psb_kernel kernel, uint32_t flags);

/* LinearBVH!(input) (src/julia/KernelInterpolation/interpolation_setup/InterpolationInput.jl:201-221):
 * Morton codes -> radix sort -> dedup -> Karras radix tree -> escape links ->
 * bottom-up AABB refit, on the device.  The device copies of all particle
 * arrays are permuted into Morton order.  perm_out[i] (host, nullable) is the
 * 0-based original index of the particle at Morton position i (enc.order - 1),
 * original meaning the order psb_set_particles was given (also when the LBVH
 * is built again without new particles: the device copies are then already in
 * Morton order, and the permutation stays relative to the caller's arrays);
 * codes_out (host, nullable) receives the sorted, de-duplicated codes.  A
 * caller that mirrors Partia's in-place contract applies perm_out to its own
 * arrays. */
int psb_build_lbvh(psb_ctx* ctx, int64_t* perm_out, uint64_t* codes_out);

/* New masses, densities and quantity columns for the particles of a built
 * LBVH, keeping the tree.  The tree depends on the coordinates and smoothing
 * lengths only, so an input whose coordinates and h still equal the LBVH's
 * leaves (matches_lbvh_leaf_order,
 * src/julia/KernelInterpolation/interpolation_setup/InterpolationInput.jl:265-267)
 * can be interpolated with that LBVH after only its values are replaced, as
 * Partia's external-LBVH driver overloads do
 * (src/julia/KernelInterpolation/grid_interpolation/drivers/PointSamples_driver.jl:98-118).
 * The arrays hold n values each in the LBVH's leaf (Morton) order, the order
 * of psb_build_lbvh's perm_out; ncol may differ from psb_set_particles'.
 * Host pointers unless PSB_FLAG_DEVICE_PTRS. */
int psb_set_values(psb_ctx* ctx, const void* m, const void* rho,
                   int32_t ncol, const void* const* cols, uint32_t flags);

/* Tree export for parity checks (LinearBVH fields,
 * src/julia/LinearBoundingVolumeHierarchy/LinearBVH/LinearBVH.jl:8-14).
 * left/right/escape/parent: 2n-1 entries each, unified 1-based ids;
 * node_min/node_max: 3*(n-1) values, axis-major (x block, y block, z block);
 * node_scale: n-1 values; root: 1 (n >= 2) or 0.  Every pointer is a host
 * pointer and may be NULL. */
int psb_get_tree(psb_ctx* ctx, int32_t* root,
                 int32_t* left, int32_t* right, int32_t* escape, int32_t* parent,
                 double* node_min, double* node_max, double* node_scale);

/* ---- interpolation -------------------------------------------------------- */

/* PointSamples_interpolation (ext/CUDAExt/KernelInterpolation/grid_interpolation/drivers/PointSamples_driver.jl:12,44;
 * CPU: src/julia/KernelInterpolation/grid_interpolation/drivers/PointSamples_driver.jl:34-48,98-118).
 * ns samples at (sx, sy, sz); out[k] receives output field k (catalog order),
 * ns values each.  hs follows hmode (NULL for PSB_H_NEAREST).  Scatter ignores
 * hmode.  Samples with no neighbour get NaN in every field
 * (general_interpolation.jl:128-131). */
int psb_interp_points(psb_ctx* ctx, int64_t ns,
                      const void* sx, const void* sy, const void* sz,
                      psb_hmode hmode, const void* hs, psb_strategy strategy,
                      const psb_catalog* cat, psb_precision prec,
                      void* const* out, uint32_t flags, psb_stats* stats);

/* StructuredGrid_interpolation for a Cartesian grid
 * (src/julia/KernelInterpolation/grid_interpolation/drivers/StructuredGrid_driver.jl:46-64):
 * the sample at linear index i + nx*(j + ny*k) is (ax[i], ay[j], az[k]),
 * Julia's column-major order (src/julia/Grids/grids/StructuredGrid.jl:115-139).
 * Coordinates are generated on the device from the axis arrays, which are
 * always host pointers (PSB_FLAG_DEVICE_PTRS applies to hs and out). */
int psb_interp_grid(psb_ctx* ctx,
                    const void* ax, int64_t nx, const void* ay, int64_t ny,
                    const void* az, int64_t nz,
                    psb_hmode hmode, const void* hs, psb_strategy strategy,
                    const psb_catalog* cat, psb_precision prec,
                    void* const* out, uint32_t flags, psb_stats* stats);

/* PointSamples(Cartesian, frame, xparams, yparams, zparams) box
 * (src/julia/Grids/grids/coordinate.jl:93-151), generated on the device:
 * frame = {x0,y0,z0, rx,ry,rz, ux,uy,uz, fx,fy,fz} (position, right, up,
 * forward in global coordinates, element type of the context);
 * params = {xmin,xmax, ymin,ymax, zmin,zmax}; sample k = i + nx*(j + ny*l).
 * frame and params are always host pointers. */
int psb_interp_box(psb_ctx* ctx, const void* frame, const void* params,
                   int64_t nx, int64_t ny, int64_t nz,
                   psb_hmode hmode, const void* hs, psb_strategy strategy,
                   const psb_catalog* cat, psb_precision prec,
                   void* const* out, uint32_t flags, psb_stats* stats);

/* LineSamples_interpolation (ext/CUDAExt/KernelInterpolation/grid_interpolation/drivers/LineSamples_driver.jl:11,49;
 * CPU: src/julia/KernelInterpolation/grid_interpolation/drivers/LineSamples_driver.jl:39-55,116-141).
 * nl lines with origins (ox,oy,oz) and unit directions (dx,dy,dz).  The
 * catalog may hold scalars only.  Partia's driver accepts PSB_SCATTER only and
 * raises ArgumentError otherwise; this returns PSB_EINVAL likewise.  The
 * gather / symmetric kernel-level variants
 * (line_integrated_scalar_interpolation.jl:76-121,168-214) are reached with
 * PSB_GATHER / PSB_SYMMETRIC plus hmode PSB_H_PER_SAMPLE or PSB_H_CONSTANT. */
int psb_interp_lines(psb_ctx* ctx, int64_t nl,
                     const void* ox, const void* oy, const void* oz,
                     const void* dx, const void* dy, const void* dz,
                     psb_hmode hmode, const void* hs, psb_strategy strategy,
                     const psb_catalog* cat, psb_precision prec,
                     void* const* out, uint32_t flags, psb_stats* stats);

/* LineSamples(Cartesian, ParallelBeam, frame, xparams, yparams)
 * (src/julia/Grids/grids/LineSamples.jl:462-486), generated on the device:
 * origins on the frame plane, every direction = frame forward.
 * params = {xmin,xmax, ymin,ymax}; line k = i + nx*j.  frame and params are
 * always host pointers. */
int psb_interp_beam(psb_ctx* ctx, const void* frame, const void* params,
                    int64_t nx, int64_t ny,
                    psb_hmode hmode, const void* hs, psb_strategy strategy,
                    const psb_catalog* cat, psb_precision prec,
                    void* const* out, uint32_t flags, psb_stats* stats);

/* _density_kernel (src/julia/KernelInterpolation/single_point_interpolation/kernels/scalar_interpolation.jl:1-75):
 * sum_b m_b W at each sample, 0 where there is no neighbour.  With
 * PSB_FLAG_NUMBER_DENSITY: _number_density_kernel (:86-166), sum_b W. */
int psb_density(psb_ctx* ctx, int64_t ns,
                const void* sx, const void* sy, const void* sz,
                psb_hmode hmode, const void* hs, psb_strategy strategy,
                psb_precision prec, void* out, uint32_t flags, psb_stats* stats);

/* Neighbour-set digest for parity: for each sample, the number of accepted
 * particles and the wrapping 64-bit sum of mix64(leaf index) over them (order
 * independent), with mix64 the SplitMix64 finaliser of the 1-based leaf index.
 * kind 0: points (a = coordinates, d ignored); kind 1: lines (a = origins,
 * d = directions).  ha_out (nullable) receives the h_a actually used. */
int psb_neighbor_digest(psb_ctx* ctx, int32_t kind, int64_t ns,
                        const void* ax, const void* ay, const void* az,
                        const void* dx, const void* dy, const void* dz,
                        psb_hmode hmode, const void* hs, psb_strategy strategy,
                        int64_t* count_out, uint64_t* hash_out, void* ha_out,
                        uint32_t flags);

/* ---- adjoint ------------------------------------------------------------------ */

/* Vector-Jacobian products of the interpolation (no counterpart in the
 * reference, which has no derivatives; they serve a ChainRulesCore.rrule of
 * PointSamples_interpolation / StructuredGrid_interpolation /
 * LineSamples_interpolation).  For the loss
 *   L = sum_k sum_s gout[k][s] * out_k(s)
 * with out_k the field k (catalog order) that the matching forward call
 * returns, they write dL/dm (gm), dL/dA (gcols[c] for particle column c; the
 * columns the catalog does not use get zeros; gcols and its entries may be
 * NULL) and dL/dx, dL/dy, dL/dz per particle, in the order the particles were
 * given to psb_set_particles.  Densities, smoothing lengths and the sample h
 * (hs, or the nearest particle's h, which is piecewise constant in the
 * positions) are held fixed.  Double particle data only (else
 * PSB_EUNSUPPORTED).  The forward sums are recomputed in PSB_PREC_FP64 where
 * the cotangents depend on them (Shepard ratios, gradients, divergences,
 * curls, or a nearest-particle h); a catalog of plain scalars (e.g. column
 * density) needs no forward pass.  The
 * pair terms are summed per particle by a traversal of an LBVH over the
 * samples (points, grids), or of the pixel lattice (beams), with the forward's
 * inclusion arithmetic: no float atomics.  Points and grids keep the
 * traversal's pair lists in a device pool of the context that grows to what
 * a call needs and stays for the next (at most 32 GiB; a call that outgrows it
 * walks again, so a context's first large call is the slowest); the results
 * do not depend on the pool's size.  gout, hs and the gradient arrays
 * are device pointers with PSB_FLAG_DEVICE_PTRS, host pointers otherwise;
 * grid axes, frame and params are host pointers. */
int psb_adjoint_points(psb_ctx* ctx, int64_t ns,
                       const void* sx, const void* sy, const void* sz,
                       psb_hmode hmode, const void* hs, psb_strategy strategy,
                       const psb_catalog* cat, const void* const* gout,
                       double* gm, double* const* gcols, double* gx, double* gy, double* gz,
                       uint32_t flags, psb_stats* stats);
int psb_adjoint_grid(psb_ctx* ctx,
                     const void* ax, int64_t nx, const void* ay, int64_t ny,
                     const void* az, int64_t nz,
                     psb_hmode hmode, const void* hs, psb_strategy strategy,
                     const psb_catalog* cat, const void* const* gout,
                     double* gm, double* const* gcols, double* gx, double* gy, double* gz,
                     uint32_t flags, psb_stats* stats);
/* Parallel-beam lines (psb_interp_beam; the frame axes must be orthonormal). */
int psb_adjoint_beam(psb_ctx* ctx, const void* frame, const void* params,
                     int64_t nx, int64_t ny,
                     psb_hmode hmode, const void* hs, psb_strategy strategy,
                     const psb_catalog* cat, const void* const* gout,
                     double* gm, double* const* gcols, double* gx, double* gy, double* gz,
                     uint32_t flags, psb_stats* stats);

/* ---- the reference's GPU design, as a baseline ------------------------------- */

/* PointSamples_interpolation with the structure of Partia's CUDA extension
 * (ext/CUDAExt/KernelInterpolation/grid_interpolation/drivers/PointSamples_driver.jl:12-27,
 *  ext/CUDAExt/KernelInterpolation/grid_interpolation/kernels/PointSamples_kernel.jl:1-68),
 * kept to measure this library against it on the same GPU; it is not the
 * library's interpolation path.  Every argument is a host array: the n
 * particles in the tree's leaf (Morton) order with ncol columns, and the tree
 * as psb_get_tree exports it (root, left and escape with unified 1-based ids,
 * axis-major node boxes, node scales), as the reference builds it on the CPU.
 * Each call copies all of it and the samples to the device, runs one thread
 * per sample in blocks of 256 (nearest-particle h by LBVH_find_nearest_h for
 * gather and symmetric, then the FP64 general interpolation kernel, each a
 * per-thread stackless DFS, no shared memory), and copies the L outputs back.
 * Device buffers are the context's and are kept between calls.  FP64 only;
 * stats->h2d_ms / interp_ms / d2h_ms split the call's event time. */
int psb_baseline_cudaext_points(psb_ctx* ctx, int64_t n,
                                const double* x, const double* y, const double* z,
                                const double* m, const double* h, const double* rho,
                                int32_t ncol, const double* const* cols, psb_kernel kernel,
                                int32_t root, const int32_t* left, const int32_t* escape,
                                const double* node_min, const double* node_max, const double* node_scale,
                                int64_t ns, const double* sx, const double* sy, const double* sz,
                                psb_strategy strategy, const psb_catalog* cat,
                                double* const* out, psb_stats* stats);

/* ---- failure injection (tests) ------------------------------------------------ */

/* No counterpart in the reference, which has no device walks to bound.  For
 * failure-detection tests: every escape link of the built LBVH that ends a
 * traversal (the right spine and the last leaf, escape 0) is pointed at the
 * root.  Node ids stay valid, so every memory access of a walk stays in
 * bounds; each walk then cycles until its step bound (4n + 8 steps), and the
 * interpolation, density, digest and adjoint calls return PSB_ETRAVERSAL.
 * psb_build_lbvh restores a correct tree.  Needs n >= 2. */
int psb_test_loop_escapes(psb_ctx* ctx);

/* No counterpart in the reference.  For tests of the point and grid adjoint
 * (psb_adjoint_points, psb_adjoint_grid): split = 1 (the default) runs them as
 * a walk that writes each tile of 32 particles' pair lists into blocks of a
 * pool, a pass that sums each block's pairs, and a pass that adds each
 * particle's block sums in the walk's order; split = 0 runs the single-kernel
 * walk, which adds the same terms in one running sum (the same values to
 * rounding).  blocks > 0 sets the pool's size for the next call (each block
 * holds 16 list entries per particle of a tile); a call whose pool runs out
 * grows it and walks again, so a small pool exercises that path and gives
 * the same bits.  split = 2 is split = 1 with a pool that keeps its size: the
 * tiles that do not fit run in the single-kernel walk. */
int psb_test_adjoint_pool(psb_ctx* ctx, int64_t blocks, int32_t split);

/* ---- interpolation without device allocation -------------------------------- */

/* No counterpart in the reference: an addition of this library.
 * psb_interp_points with PSB_FLAG_DEVICE_PTRS semantics (sx, sy, sz, hs and
 * every out[k] are device pointers) that allocates no device memory.  It is
 * for callers that cannot allocate while they interpolate: a host whose device
 * memory is held by another framework's caching pool, where a cudaMalloc in
 * mid-step can fail; a pipeline with a memory budget fixed at start-up; a
 * caller that cannot take the device-wide synchronisation of a cudaFree.  Its
 * per-call scratch (sample Morton order and counters) is one file-scope device
 * array of PSB_NOALLOC_SCRATCH_BYTES, resident on every GPU that loads the
 * library.
 *  - ns <= PSB_NOALLOC_MAX_SAMPLES, else PSB_EINVAL (split the call);
 *  - the first call on a device looks the array's address up once, with that
 *    device current (again after a cudaDeviceReset gives the device a new
 *    context); make that first call before any stream capture begins;
 *  - all calls on a device share the array: calls whose GPU work overlaps
 *    (several streams or contexts on one device) race and must be serialised
 *    by the caller;
 *  - particles and LBVH must already be on the device (psb_set_particles and
 *    psb_build_lbvh allocate; this call does not).
 * It runs the single-kernel form of the point interpolation
 * (PSB_FLAG_SINGLE_KERNEL), so its results agree with psb_interp_points' to
 * rounding. */
#define PSB_NOALLOC_MAX_SAMPLES 262144
#define PSB_NOALLOC_SCRATCH_BYTES (8u << 20)
int psb_interp_points_noalloc(psb_ctx* ctx, int64_t ns,
                              const void* sx, const void* sy, const void* sz,
                              psb_hmode hmode, const void* hs, psb_strategy strategy,
                              const psb_catalog* cat, psb_precision prec,
                              void* const* out, psb_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* PARTIA_B200_H */
