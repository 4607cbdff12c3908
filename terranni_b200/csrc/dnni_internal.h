// dnni_internal.h -- context layout shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <string>

#include "../../include/dnni.h"
#include "dnni_kernels.cuh"

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};

struct dnni_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    dnni_settings s{};
    // per-work-package scratch (grow-only until dnni_clear)
    DevBuf rank, sorted, cnt, start, bsum, pix, D, Dc, bmask, smask, far, rownear, near;
    // staging for the host-buffer entry point
    DevBuf in_xyz, in_gid, out_h, out_site;
    dnni::Scalars* d_sc = nullptr;
    dnni::Scalars* h_sc = nullptr;   // pinned mirror
    cudaEvent_t ev[6] = {};
    std::string err;
    size_t held = 0;
    double acc_ms[4] = {};
    int64_t calls = 0;
};

dnni_status dnni_ensure(dnni_ctx* c, DevBuf& b, size_t bytes);
void dnni_release(DevBuf& b, dnni_ctx* c);
void dnni_free_all(dnni_ctx* c);
dnni_status dnni_tile_geometry(dnni_ctx* c, const dnni_workpackage* wp, int64_t n, dnni::TileParams& t);
void dnni_bin_grid(const dnni_ctx* c, const int32_t bbox[6], int64_t n, dnni::TileParams& t);
dnni_status dnni_run_device(dnni_ctx* c, const dnni_workpackage* wp, const int32_t* d_xyz, const uint32_t* d_gid,
                            int64_t n, float* d_h, uint32_t* d_site, cudaStream_t st, dnni_stats* stats);
