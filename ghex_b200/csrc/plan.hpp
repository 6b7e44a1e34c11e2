// Exchange plans: the work-descriptor table of one field set, its tiles, device copies and the
// captured CUDA graph of the batched form.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "bulk.hpp"
#include "core.hpp"
#include "exchange.hpp"
#include "staged.hpp"

struct ghexb_plan_s
{
    ghexb_context_s* ctx = nullptr;
    std::vector<ghexb_field_s> fields;
    // unstructured in-place receive (unstructured/communication_object_ipr.hpp:127-141): the
    // values received from a neighbour land on consecutive halo rows from its first receive index
    bool in_place_receive = false;
    // Sharded exchange (one process per GPU): `fields` holds every domain's fields, those of other
    // processes mapped from their memory, and shard_local[slot] marks this process's own. mode 0:
    // every descriptor; 1 (pull): the descriptors that write a local field, reading peers'
    // interiors; 2 (push): those that read a local field, writing peers' halos, whose adjoint
    // gathers every image of the local owners (the pull form has no adjoint: a remote owner's
    // images lie in several processes' plans).
    int shard_mode = 0;
    std::vector<char> shard_local;

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
    std::vector<int64_t> box_src_off, box_dst_off; // byte offsets of descriptor pointers from their fields' data
    std::vector<int64_t> list_src_off, list_dst_off;
    std::vector<int64_t> adj_src_off, adj_dst_off;
    int n_logical = 0;

    // Forward work (exchange.cu), one CTA per tile: xf is the batched form's table (the most
    // DRAM bytes per element first), xp the per-field form's (grouped by logical field) and xb
    // the per-box form's (grouped by descriptor).
    std::vector<ghexb::xtile> xf, xp, xb;
    // Index blocks of the list tiles, one per tile of xf, xp and xb (exchange.hpp
    // k_block_ints each): the indices of the tile's columns, loaded beside its record. Empty
    // when the plan has no lists.
    std::vector<int32_t> xf_blk, xp_blk, xb_blk;
    // Bulk column tiles of the batched form (bulk.hpp): of the list descriptors in 16-byte units
    // between device fields, those with index i % 4 < bulk_share move by the copy engine (the bulk
    // kernel, beside the element kernel on a second stream when both have work) instead of the
    // element kernel: 0 none, 4 all; chosen by the autotuner. bt_blk holds each tile's index block;
    // bt_list and bt_col0 (host only) its list and first column.
    int bulk_share = 4;
    std::vector<ghexb::btile> bt;
    std::vector<int32_t> bt_blk;
    std::vector<int> bt_list, bt_col0;
    ghexb::btile* d_bt = nullptr;
    int32_t* d_bt_blk = nullptr;
    size_t cap_bt = 0, cap_bt_blk = 0;
    // tensor maps of the bulk tiles' fields (a row per index, the levels of a column in a row),
    // for their four-column gather and scatter copies, and their geometry for the host replay
    struct bmap_info
    {
        const char* base;
        int64_t rows, stride; // rows (indices) and bytes per row step
        int width, es;        // elements per row moved (the column), element size
    };
    std::vector<CUtensorMap> bmaps;
    std::vector<bmap_info> bmap_geo;
    CUtensorMap* d_bmaps = nullptr;
    size_t cap_bmaps = 0;
    bool forms_stale = false; // xp and xb moved on the host by a rebind, not yet on the device
    int32_t *d_xf_blk = nullptr, *d_xp_blk = nullptr, *d_xb_blk = nullptr;
    size_t cap_xf_blk = 0, cap_xp_blk = 0, cap_xb_blk = 0;
    // x-face boxes whose rows interleave (A's row r ends where B's row r + 1 begins): the
    // batched and per-field tables move each pair as one set of contiguous segments
    std::vector<std::pair<int, int>> pairs; // (A, B) box indices
    std::vector<int> box_pair;              // per box: its pair, or -1
    std::vector<ghexb::xtile> xpair;        // host only: the pairs' tiles, for the replay check
    std::vector<std::pair<int, int>> xpair_range;
    std::vector<std::pair<int, int>> xp_field;          // [begin, count) in xp per logical field
    std::vector<std::pair<int, int>> xb_box, xb_list;   // [begin, count) in xb per descriptor
    // Box adjoint in gather form (gather_ok), else by conflict-free phases of the box descriptors.
    bool gather_ok = false;
    std::string gather_reason;
    std::vector<ghexb::gcell> cells;
    // Unstructured adjoint in gather form (list_gather_ok), else by phases: every owner column
    // with its ordered image columns, grouped by (element size, images, levels, level strides).
    struct list_owner
    {
        int slot;
        int64_t off; // byte offset of the owner column from its field's data
        int32_t levels, s_ls, d_ls;
        int esize, nimg;
        int img_slot[ghexb::k_max_images];
        int64_t img_off[ghexb::k_max_images];
    };
    bool list_gather_ok = false;
    std::vector<list_owner> lowners;
    std::vector<uint64_t> lcols; // column table of the owner groups (addresses of the columns)
    // per unstructured gather tile (after the gt_boxes box cells): its slice of lcols in a block
    // of k_gblock_entries, flagged in the tile's pad[0] when the slice fits
    std::vector<uint64_t> gblk;
    uint64_t* d_gblk = nullptr;
    size_t cap_gblk = 0;
    std::vector<ghexb::gtile> gt; // box cells first (gt_boxes of them), then unstructured owner groups
    int gt_boxes = 0;
    // adjoint tiles of the phased kernels (boxes when !gather_ok, lists) grouped by phase
    std::vector<ghexb::tile> adj_btiles, adj_ltiles;
    std::vector<std::pair<int, int>> adj_bphase_range, adj_lphase_range;
    std::vector<int> box_phase, list_phase;

    // device copies
    ghexb::box_desc* d_boxes = nullptr;
    ghexb::list_desc* d_lists = nullptr;
    ghexb::list_desc* d_adj_lists = nullptr;
    int32_t* d_idx = nullptr;
    ghexb::xtile* d_xf = nullptr;
    ghexb::xtile* d_xp = nullptr;
    ghexb::xtile* d_xb = nullptr;
    ghexb::gtile* d_gt = nullptr;
    uint64_t* d_lcols = nullptr;
    size_t cap_xf = 0, cap_xp = 0, cap_xb = 0, cap_gt = 0, cap_lcols = 0; // elements allocated behind the tables
    ghexb::tile* d_adj_btiles = nullptr;
    ghexb::tile* d_adj_ltiles = nullptr;
    unsigned* d_counters = nullptr; // tile scheduler counters of the phased adjoint kernels

    int64_t num_tiles() const; // non-empty tiles of the batched table
    int adjoint_launches() const;

    // statistics
    int64_t halo_elements = 0;
    int64_t algorithmic_bytes = 0;
    int64_t index_bytes = 0;
    bool adjoint_ok = true;
    std::string adjoint_reason;

    // tuning: elements per thread (4, 8 or 16) and threads per CTA of the forward kernel
    int per_thread = 8;
    int block = 256;
    bool use_pairs = true; // batched and per-field tables move x-face pairs as segments
    // adjoint gather tiles of short rows: -1 half the size, 0 sized by row length, 1 and 2 that
    // size doubled or quadrupled (never beyond a full tile); chosen by the autotuner
    int gather_scale = 0;
    // Unstructured adjoint in bulk form (bulk.hpp): of every owner group whose columns are
    // contiguous and 16-byte aligned, the first gather_bulk quarters of the owners go to the bulk
    // gather kernel, beside list_gather_kernel on a second stream; chosen by the autotuner.
    // bgt_blk: per tile its column addresses; bgt_first (host only): its first owner in lowners.
    int gather_bulk = 0;
    std::vector<ghexb::bgtile> bgt;
    std::vector<uint64_t> bgt_blk;
    std::vector<int> bgt_first;
    ghexb::bgtile* d_bgt = nullptr;
    uint64_t* d_bgt_blk = nullptr;
    size_t cap_bgt = 0, cap_bgt_blk = 0;

    // Staged form of box descriptors (staged.hpp), batched form only: the boxes marked in
    // box_staged are loaded through tensor maps by the staged kernel, which runs beside the
    // element kernel (its tiles are then the other boxes, the pairs of unstaged boxes and the
    // lists). staged_mode 0: none; 1: boxes of rows of at most 64 bytes and boxes whose source
    // rows run along the destination's second axis; 2: every box a tensor map can load.
    int staged_mode = 0;
    int stage_bytes = 16384, stages = 8, stage_consumers = 4, stage_ctas_per_sm = 1;
    std::vector<char> box_staged;
    std::vector<char> field_on_device; // per field: device memory (set when the plan is uploaded)
    bool encode_maps = true;           // false for host-only checks: geometry without tensor maps
    struct smap_info // host copy of a tensor map's geometry, for the replay check
    {
        const char* base;
        int64_t dims[3], strides[2]; // elements; byte strides of dimensions 1 and 2
        int es, w, h, d;             // element size, load box
        int slot;                    // source field slot
    };
    std::vector<CUtensorMap> smaps;
    std::vector<smap_info> smap_host;
    std::vector<ghexb::sitem> sitems;
    std::vector<int> sitem_box; // per item: its box descriptor
    CUtensorMap* d_smaps = nullptr;
    ghexb::sitem* d_sitems = nullptr;
    unsigned* d_status = nullptr;
    size_t cap_smaps = 0, cap_sitems = 0;
    cudaStream_t side_stream = nullptr;
    cudaEvent_t fork_event = nullptr, join_event = nullptr;
    // Page-locked staging of the table uploads (plan.cu host_stager): copies never read the
    // library's pageable heap memory, which may share pages with host fields that the page
    // registry has locked (a copy whose source straddles a locked range is refused by CUDA).
    // A ring of four buffers, each reused once the copies out of its previous use are done.
    struct stage_buffer
    {
        void* ptr = nullptr;
        size_t cap = 0;
        cudaEvent_t done = nullptr;
    };
    stage_buffer h_stage[4];
    int h_stage_next = 0;

    // graphs of the batched form and of the adjoint, captured on first use
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t adj_graph = nullptr;
    cudaGraphExec_t adj_exec = nullptr;

    ~ghexb_plan_s();
};

namespace ghexb
{
// Builds the host tables of a plan from the fields (plan.cu). Throws ghexb::error.
void build_tables(ghexb_plan_s& plan, ghexb_context_s* ctx, const ghexb_field* fields, int n);
// Kernels address a field's memory directly: device or managed memory, or pinned host memory
// mapped at the same address (unified addressing; the kernels then move its bytes over the host
// interconnect). Anything else is refused before a launch could touch it.
void check_accessible(const void* p);
// ... every page of [p, p + bytes) when it is host memory
void check_accessible(const void* p, size_t bytes);
// bytes from a field's data pointer to one past its last element
size_t field_bytes(const ghexb_field_s& f);
// Uploads the tables and tiles to the device.
void upload_plan(ghexb_plan_s& plan);
// build_tables + upload_plan
void build_plan(ghexb_plan_s& plan, ghexb_context_s* ctx, const ghexb_field* fields, int n);
// Replays on the host the address computation of every element the forward and adjoint kernels
// touch and checks it against the memory span of its field; returns the number of elements.
int64_t check_tables(ghexb_plan_s& plan);
// Host-only: the tile tables moved to other field memory by a rebind equal the tables built there.
void check_relocation(ghexb_plan_s& plan);
// Host-only: forward tiles of the current tuning and the adjoint tiles, addressing the fields'
// current data; list tiles point into `idx` (the device copy of plan.idx, or any copy of it).
void build_tiles(ghexb_plan_s& plan, const int32_t* idx);
// build_tiles + copy of the tile tables to the device on `stream` (allocating only when they grew).
void retile(ghexb_plan_s& plan, cudaStream_t stream = nullptr);
void release_graph(ghexb_plan_s& plan);
void launch_plan(ghexb_plan_s& plan, int form, cudaStream_t stream);
void graph_launch_plan(ghexb_plan_s& plan, cudaStream_t stream);
void adjoint_plan(ghexb_plan_s& plan, cudaStream_t stream);
void autotune_plan(ghexb_plan_s& plan, cudaStream_t stream, int repeats);
// Moves the plan to new field memory of the same layout (one pointer per field, in plan order):
// recomputes the descriptor pointers and rewrites the device tables on `stream`.
void rebind_plan(ghexb_plan_s& plan, void* const* data, int n, cudaStream_t stream);
void check_cuda(cudaError_t e, const char* what);
// Host-only: decides which boxes the staged kernel takes (plan.staged_mode) and builds their
// tensor maps and items (staged_plan.cu).
void build_staged(ghexb_plan_s& plan);
// Host replay of every staged item's element: the load coordinates stay inside the map, the
// source and destination inside their fields, and the items move exactly their boxes' elements.
// Returns the elements checked.
int64_t check_staged(const ghexb_plan_s& plan);
// The staged kernel of the batched form on a side stream forked from and joined to `stream`.
void launch_staged_plan(ghexb_plan_s& plan, cudaStream_t stream);
// The second stream of the batched form and its fork and join events, made on first use.
void ensure_side_stream(ghexb_plan_s& plan);
// Host-only: the least DRAM traffic of one exchange with a cold cache at the given sector size:
// every sector holding a source element is read, every sector holding a destination element is
// written back, and a sector written in part that holds no source element is read first.
void dram_floor(const ghexb_plan_s& plan, int sector, int64_t& read_bytes, int64_t& write_bytes);
// Records a failure for ghexb_last_error() (capi.cu).
int set_last_error(int code, const std::string& msg);
} // namespace ghexb
