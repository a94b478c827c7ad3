// psb_ctx.hpp -- host-side context of the C ABI (device buffers, stream, errors).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <unordered_map>
#include <vector>

#include "psb_common.cuh"

struct psb_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;

    // particles (device, Morton order after a build); element size es
    int64_t n = 0;
    psb_dtype dt = PSB_F64;
    psb_kernel kern = PSB_KERNEL_M4;
    size_t es = 8;
    int32_t ncol = 0;
    void* x = nullptr; void* y = nullptr; void* z = nullptr;
    void* m = nullptr; void* h = nullptr; void* rho = nullptr;
    std::vector<void*> cols;        // ncol column buffers (taken from colpool)
    std::vector<void*> colpool;     // column buffers kept across set_particles calls
    std::vector<size_t> colcap;     // their sizes in bytes
    void** d_cols = nullptr;

    // LBVH
    bool built = false;
    int32_t root = 0;
    uint64_t* codes = nullptr;
    int64_t* order = nullptr;       // caller's index (as given to psb_set_particles) of each Morton position
    bool order_fresh = true;        // device arrays still in the caller's order (no build since set_particles)
    int32_t* left = nullptr; int32_t* right = nullptr;
    int32_t* escape = nullptr; int32_t* parent = nullptr;
    int32_t* range_lo = nullptr; int32_t* range_hi = nullptr;
    int4* links = nullptr;
    void* nmin[3] = {nullptr, nullptr, nullptr};
    void* nmax[3] = {nullptr, nullptr, nullptr};
    void* nscale = nullptr;
    float4* node_lo = nullptr; float4* node_hi = nullptr; float4* leaf4 = nullptr;
    float* mrho = nullptr; float* mf = nullptr;
    float4* leafK = nullptr;  // per leaf (1/h, sigma/h^3, sigma/h^4, m/rho), float
    float2* spanb = nullptr;  // at a span's first leaf: (max |leaf4.xyz|_1, max h) over the span, rounded up
    float* colsf = nullptr;  // float copies of the columns (double inputs), ncol x n
    int32_t* sfirst = nullptr;  // first leaf of each leaf's span (double inputs)
    float* colsr = nullptr;  // columns relative to the span's first leaf, A[i] - A[sfirst[i]] in float, ncol x n
    float coord_err = 0.f;
    double bbox[6] = {0, 0, 0, 0, 0, 0};  // particle min x,y,z, max x,y,z

    unsigned* d_err = nullptr;  // device error word
    double* lut_d = nullptr;    // line-integrated kernel table of the context's kernel (4096, double)
    float* lut_f = nullptr;     // the same table rounded to float
    float* lut_fs = nullptr;    // a 1000-entry float table of the same integral (PSB_FLAG_LUT1000_F32)
    int lut_kern = -1;          // kernel family of the tables above

    // reusable scratch (grown on demand, freed with the context)
    struct Slot { void* p = nullptr; size_t bytes = 0; };
    Slot scratch[96];
    // sizes of the particle and tree buffers above, keyed by the address of
    // the pointer member: they are kept across set_particles and builds and
    // reallocated only to grow, so repeated builds of the same size (the
    // sample LBVH of every adjoint call) allocate nothing
    std::unordered_map<const void*, size_t> caps;

    // adjoint: while adj_lam is set, an FP64 interpolation call writes the
    // cotangents of its per-sample sums (from the output cotangents adj_gout,
    // a device array of L device pointers) to adj_lam and h_a to adj_ha,
    // instead of output fields
    const double* const* adj_gout = nullptr;
    double* adj_lam = nullptr;
    int64_t adj_lam_stride = 0;
    void* adj_ha = nullptr;
    struct psb_ctx* sctx = nullptr;  // LBVH over the samples of the last adjoint call
    int64_t adj_blocks = 0;           // list-block pool of the two-kernel point adjoint (grown to the last need)
    int adj_split = 1;                // 0: k_adj_points alone; 2: the pool keeps its size (psb_test_adjoint_pool)

    cudaEvent_t ev[8] = {};
    // copy streams (in, out) and three more compute streams of the chunked
    // host-memory path (created on first use)
    cudaStream_t cstream[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t pev[16] = {};
    // the other streams of the two-kernel point path (batches spread over them)
    cudaStream_t sstream[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t sev[4] = {};
};

namespace psb {

// The context's device for the duration of an entry point; the caller's
// current device is restored on return.
struct DeviceGuard {
    int prev = -1, dev;
    explicit DeviceGuard(int d) : dev(d) {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            cudaGetLastError();
            prev = -1;
        }
        if (prev != dev) err = cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    }
    cudaError_t err = cudaSuccess;
};

// Record an error message on the context and return the code.
int fail(psb_ctx* c, int code, const std::string& msg);
// PSB_ETRAVERSAL with the message of a nonzero device error word (read back
// after a call's kernels; the caller clears the word).
int device_error(psb_ctx* c, unsigned herr);
// Translate a CUDA error into PSB_ECUDA (or PSB_ENOMEM) with a message.
int cuda_fail(psb_ctx* c, cudaError_t e, const char* what);
// Grow-on-demand scratch slot k to at least `bytes`; returns nullptr on failure.
void* scratch(psb_ctx* c, int k, size_t bytes);
// With PSB_FLAG_DEVICE_PTRS the kernels read or write a caller's pointer
// directly, so it must be reachable from the context's device: device memory
// of that device, managed memory, or page-locked host memory mapped at the
// same address.  Anything else (pageable host memory, another device's
// memory) would fault inside a kernel; it is refused here with PSB_EINVAL.
// A null pointer passes (the callers check for NULL where it matters).
int check_device_ptr(psb_ctx* c, const void* p, const char* what);
// Device buffer *p with room for at least `bytes`, reallocated only when it
// must grow (after the context's stream has finished with the old one).
cudaError_t dgrow(psb_ctx* c, void** p, size_t bytes);
template <class P> cudaError_t dgrow_t(psb_ctx* c, P** p, size_t bytes) { return dgrow(c, (void**)p, bytes); }
// Mark the LBVH as absent (its buffers are kept for the next build).
void reset_tree(psb_ctx* c);
// Free every particle and tree buffer (context destruction).
void release_buffers(psb_ctx* c);

// build.cu
int build_lbvh(psb_ctx* c);
// Re-derive the leaf records that depend on m, rho and the columns (after a
// values-only update of a built LBVH); queued on the context stream.
int repack_values(psb_ctx* c);
// Test hook: turn every end-of-walk escape link into a link to the root.
int loop_escapes(psb_ctx* c);

// scan.cu helpers used by the build and the interpolation drivers
cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, psb_ctx* c, int slot_base);
cudaError_t inclusive_max_scan_i64(int64_t* data, int64_t n, psb_ctx* c, int slot_base);
// Stable LSD radix sort (onesweep, 8-bit digits) of (key, value) pairs,
// results in keys/vals; scratch slot slot_base.  skip_constant_digits: read
// back which digits vary (one host sync) and sort only those; otherwise all
// eight passes run without a host round trip.  A look-back wait that runs
// out sets PSB_DERR_SORT in the context's error word.
// key_bits: the keys are below 2^key_bits (the digits above are not sorted).
cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, int64_t n, psb_ctx* c, int slot_base, int* launches,
                             bool skip_constant_digits = true, int key_bits = 64);
// The same sort on caller-provided scratch of at least
// radix_sort_pairs_scratch_bytes(n) bytes (256-byte aligned); allocates nothing.
size_t radix_sort_pairs_scratch_bytes(int64_t n);
cudaError_t radix_sort_pairs_in(uint64_t* keys, uint32_t* vals, int64_t n, void* scratch_space, size_t bytes,
                                cudaStream_t s, unsigned* err, int* launches);

template <class T> TreeView<T> tree_view(psb_ctx* c);

}  // namespace psb

#define PSB_CUDA_TRY(ctx, call, what)                         \
    do {                                                      \
        cudaError_t _e = (call);                              \
        if (_e != cudaSuccess) return psb::cuda_fail(ctx, _e, what); \
    } while (0)
