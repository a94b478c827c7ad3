// psb_host.hpp -- internal host interface between the C ABI and the drivers.
#pragma once

#include "interp.cuh"
#include "psb_ctx.hpp"

namespace psb {

struct SampleReq {
    int kind = SRC_ARRAYS;
    bool line = false;
    int64_t ns = 0;
    const void* a[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    const void* ax = nullptr; const void* ay = nullptr; const void* az = nullptr;
    int64_t nx = 0, ny = 0, nz = 0;
    const void* frame = nullptr;
    const void* params = nullptr;
};

int run(psb_ctx* c, const SampleReq& rq, int hmode, const void* hs, int st, const psb_catalog* cat, int prec,
        void* const* out, uint32_t flags, psb_stats* stats, int what, int64_t* dcount, uint64_t* dhash, void* ha_out);

// M4 line-integrated table on the reference grid Q_k = (k-1) 2/4095
// (table/line_integrated_kernel_tables.jl:1,1029), regenerated by quadrature.
void line_table(int kernel, double* I, int n);

}  // namespace psb
