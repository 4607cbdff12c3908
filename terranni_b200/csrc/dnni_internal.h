// dnni_internal.h -- context and batch layout shared by the engine's
// translation units.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dnni.h"
#include "dnni_kernels.cuh"
#include "dnni_plan.h"

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};

// Device scratch of one batch (or of the context's single work packages);
// `list` serves only the reference-default mode (its per-tile point lists).
struct Scratch {
    DevBuf sorted, list, cnt, start, bsum, bmask, smask, rownear, near, pix, far, D, Dc, sc, ctr, tables;
};

// Raw device pointers of a scratch set for one launch sequence.
struct DevArrays {
    int4* sorted = nullptr;
    int* cnt = nullptr;
    int* start = nullptr;
    int* bsum = nullptr;
    uint64_t* bmask = nullptr;
    uint64_t* smask = nullptr;
    int* rownear = nullptr;
    int64_t* near = nullptr;
    int2* pix = nullptr;
    dnni::FarSlot* far = nullptr;
    unsigned long long* D = nullptr;
    int* Dc = nullptr;
    dnni::Scalars* sc = nullptr;
    dnni::BatchCounters* ctr = nullptr;
    unsigned char* tables = nullptr;
};

struct dnni_ctx;

// Device buffers of the segment driver and the server's resident cloud.
struct SegBufs {
    DevBuf xin, sxyz, sgid, part, cur, cnt, start, bbox, occ, gxyz, ggid, gout[2], gsite[2], chunks, ring;
    void release(dnni_ctx* c);
};

// Device buffers of the space-time driver (grow-only until dnni_clear).
struct StBufs {
    DevBuf xin, tin, xyz, idx, gs, site, pix;
    Scratch scr;                     // the per-time-value batch
};

struct dnni_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    dnni_settings s{};
    Scratch scr;                     // single work packages (grow-only until dnni_clear)
    SegBufs seg;                     // segment driver buffers (grow-only until dnni_clear)
    Scratch seg_scr;
    StBufs st;
    DevBuf in_xyz, in_gid, out_h, out_site;   // staging for the host-buffer entry point
    unsigned char* h_tables = nullptr;        // pinned staging of the tile tables
    size_t h_tables_cap = 0;
    dnni::Scalars* h_sc = nullptr;            // pinned mirror of one tile's scalars
    dnni::BatchCounters* h_ctr = nullptr;
    cudaEvent_t ev[6] = {};
    std::string err;
    size_t held = 0;
    double acc_ms[4] = {};
    int64_t calls = 0;
};

// A slice of a batch for the pipelined host-buffer run: tiles whose point
// rows form one range, so that the slice's upload, launch sequence and
// download can overlap those of its neighbours.
struct BatchSlice {
    dnni::HostBatch hb;
    DevBuf tables;
    dnni::BatchTables bt{};
    DevArrays arr;                       // the slice's own part of the batch's scratch
    int64_t row0 = 0, row1 = 0, out0 = 0, out1 = 0, site0 = 0, site1 = 0;
};

struct dnni_batch {
    dnni_ctx* ctx = nullptr;
    std::vector<dnni_tile> tiles_in;     // the caller's tiles, for slicing
    dnni_batch_options opt{};
    std::vector<BatchSlice> slices;      // planned on the first host-buffer run
    bool sliced = false, slices_planned = false;
    cudaStream_t s_in = nullptr, s_out = nullptr, s_cmp = nullptr;   // s_cmp: the second compute stream
    DevBuf slice_ctrs;                   // one BatchCounters per slice
    std::vector<cudaEvent_t> ev_in, ev_done;
    dnni::BatchCounters* h_ctrs = nullptr;
    dnni::HostBatch hb;
    Scratch scr;
    DevArrays arr;
    dnni::BatchTables bt{};
    std::vector<int> order;          // batch position -> caller's tile index
    int use_graph = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* graph_key[4] = {};   // pointers the captured graph was built for
    cudaStream_t graph_stream = nullptr;
    DevBuf in_xyz, in_gid, out_h, out_site;
    std::vector<dnni::Scalars> h_sc;
};

dnni_status dnni_ensure(dnni_ctx* c, DevBuf& b, size_t bytes);
void dnni_release(DevBuf& b, dnni_ctx* c);
void dnni_free_all(dnni_ctx* c);
