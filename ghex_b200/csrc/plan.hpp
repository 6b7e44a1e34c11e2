// Exchange plans: the work-descriptor table of one field set, its tiles, device copies and the
// captured CUDA graph of the batched form.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "core.hpp"

struct ghexb_plan_s
{
    ghexb_context_s* ctx = nullptr;
    std::vector<ghexb_field_s> fields;

    // host tables
    std::vector<ghexb::box_desc> boxes;
    std::vector<ghexb::list_desc> lists;     // forward (16-byte units where aligned)
    std::vector<ghexb::list_desc> adj_lists; // adjoint (element units, distinct owners)
    std::vector<int64_t> list_idx_off;       // per forward list: offset of (sidx, didx) in idx
    std::vector<int64_t> adj_idx_off;        // per adjoint list: offset of its sidx in idx
    std::vector<int64_t> adj_didx_off;       // per adjoint list: offset of its didx in idx
    std::vector<int32_t> idx;
    std::vector<int> box_src_slot, box_dst_slot;   // field slots of each box descriptor
    std::vector<int> list_src_slot, list_dst_slot; // field slots of each forward list descriptor
    std::vector<int> adj_src_slot, adj_dst_slot;   // field slots of each adjoint list descriptor
    int n_logical = 0;

    // Forward tiles in four classes, each with its own kernel instance: box descriptors of 8/4-byte
    // and of 2/1-byte elements, list descriptors of 16/8-byte and of 4/2/1-byte units. Within a
    // class, tiles are grouped by logical field, then by descriptor.
    // ftiles: the batched form's table, most expensive tiles first (dynamic scheduling then fills
    // the tail with cheap ones); ptiles: the same tiles grouped by logical field for the per-field
    // and per-box forms.
    static constexpr int k_classes = 4;
    std::vector<ghexb::tile> ftiles[k_classes];
    std::vector<ghexb::tile> ptiles[k_classes];
    std::vector<std::pair<int, int>> logical_range[k_classes]; // [begin, count) in ptiles per logical field
    std::vector<std::pair<int, int>> box_range, list_range;    // [begin, count) in ptiles per descriptor
    // adjoint tiles (box, list) grouped by phase
    std::vector<ghexb::tile> adj_btiles, adj_ltiles;
    std::vector<std::pair<int, int>> adj_bphase_range, adj_lphase_range;
    std::vector<int> box_phase, list_phase;

    // device copies
    ghexb::box_desc* d_boxes = nullptr;
    ghexb::list_desc* d_lists = nullptr;
    ghexb::list_desc* d_adj_lists = nullptr;
    int32_t* d_idx = nullptr;
    ghexb::tile* d_ftiles[k_classes] = {nullptr, nullptr, nullptr, nullptr};
    ghexb::tile* d_ptiles[k_classes] = {nullptr, nullptr, nullptr, nullptr};
    ghexb::tile* d_adj_btiles = nullptr;
    ghexb::tile* d_adj_ltiles = nullptr;
    unsigned* d_counters = nullptr; // tile scheduler counters, two per tile class

    int64_t num_tiles() const
    {
        int64_t n = 0;
        for (const auto& t : ftiles) n += (int64_t)t.size();
        return n;
    }

    // statistics
    int64_t halo_elements = 0;
    int64_t algorithmic_bytes = 0;
    int64_t index_bytes = 0;
    bool adjoint_ok = true;
    std::string adjoint_reason;

    // tuning
    int tile_elems = 8192;
    int block = 256;
    int ctas_per_sm = 4;

    // graph of the batched form
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    ~ghexb_plan_s();
    int grid(int ntiles) const;
};

namespace ghexb
{
// Builds the host tables of a plan from the fields (plan.cu). Throws ghexb::error.
void build_tables(ghexb_plan_s& plan, ghexb_context_s* ctx, const ghexb_field* fields, int n);
// Uploads the tables and tiles to the device.
void upload_plan(ghexb_plan_s& plan);
// build_tables + upload_plan
void build_plan(ghexb_plan_s& plan, ghexb_context_s* ctx, const ghexb_field* fields, int n);
// Replays on the host the address computation of every element the forward and adjoint kernels
// touch and checks it against the memory span of its field; returns the number of elements.
int64_t check_tables(const ghexb_plan_s& plan);
// Host-only: tile tables of the current tuning (no device memory touched).
void build_tiles(ghexb_plan_s& plan);
// build_tiles + upload of the tile tables.
void retile(ghexb_plan_s& plan);
void release_graph(ghexb_plan_s& plan);
void launch_plan(ghexb_plan_s& plan, int form, cudaStream_t stream);
void graph_launch_plan(ghexb_plan_s& plan, cudaStream_t stream);
void adjoint_plan(ghexb_plan_s& plan, cudaStream_t stream);
void autotune_plan(ghexb_plan_s& plan, cudaStream_t stream, int repeats);
void check_cuda(cudaError_t e, const char* what);
// Records a failure for ghexb_last_error() (capi.cu).
int set_last_error(int code, const std::string& msg);
} // namespace ghexb
