/*
 * ghex_b200 C ABI — B200-native halo exchange for many sub-domains resident on one GPU.
 *
 * Every entry point returns an int status (GHEXB_OK == 0). On failure the message is
 * kept per thread and read with ghexb_last_error(). All handles are opaque; all
 * sizes and coordinates are plain ints; data pointers are device pointers of the
 * current CUDA device; streams are cudaStream_t passed as void*.
 *
 * Each group below names the GHEX interface it replaces (paths relative to the
 * GHEX source tree, version 0.4.0).
 */
#ifndef GHEX_B200_H
#define GHEX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------- */
#define GHEXB_OK 0
#define GHEXB_ERR_INVALID 1      /* bad argument (null pointer, negative size, bad dtype ...) */
#define GHEXB_ERR_CUDA 2         /* a CUDA runtime call failed */
#define GHEXB_ERR_BUSY 3         /* "earlier exchange operation was not finished"
                                    (communication_object.hpp:360,401) */
#define GHEXB_ERR_INCOMPATIBLE 4 /* "field incompatible with available domains!"
                                    (pattern_container.hpp:94), dtype/component mismatch */
#define GHEXB_ERR_RANGE 5        /* a halo box or index falls outside the wrapped memory */
#define GHEXB_ERR_ALLOC 6        /* device or host allocation failed */
#define GHEXB_ERR_INTERNAL 7

/* ---- element types (bitwise copies; negation/addition only for float types) ---------- */
#define GHEXB_F32 0
#define GHEXB_F64 1
#define GHEXB_I32 2
#define GHEXB_I64 3
#define GHEXB_U8 4
#define GHEXB_U16 5

/* ---- exchange forms for ghexb_plan_launch -------------------------------------------- */
#define GHEXB_FORM_BATCHED 0   /* one kernel walks the whole descriptor table */
#define GHEXB_FORM_PER_FIELD 1 /* one kernel launch per field */
#define GHEXB_FORM_PER_BOX 2   /* one kernel launch per field per iteration space, the launch
                                  granularity of serialization<gpu>::pack/unpack
                                  (structured/pack_kernels.hpp:196-215) */

typedef struct ghexb_context_s* ghexb_context;
typedef struct ghexb_pattern_s* ghexb_pattern;
typedef struct ghexb_field_s* ghexb_field; /* a field bound to a pattern: GHEX's buffer_info */
typedef struct ghexb_co_s* ghexb_co;
typedef struct ghexb_handle_s* ghexb_handle;
typedef struct ghexb_plan_s* ghexb_plan;

typedef struct ghexb_plan_info_t
{
    int64_t num_fields;        /* fields given to the plan */
    int64_t num_descriptors;   /* box or index-list work descriptors */
    int64_t num_tiles;         /* tiles of the batched kernel */
    int64_t halo_elements;     /* halo elements written per exchange */
    int64_t algorithmic_bytes; /* sum over halo elements of sizeof(T) * (1 read + 1 write) */
    int64_t index_bytes;       /* bytes of index lists read per exchange (unstructured) */
    int64_t adjoint_launches;  /* kernel launches of one adjoint */
    int64_t adjoint_cells;     /* owner cells of the gather-form box adjoint (0: phased form) */
    int32_t elems_per_thread;  /* current tuning: elements a thread moves (4, 8 or 16) */
    int32_t block;             /* current tuning: threads per CTA */
    int32_t grid;              /* CTAs of the batched launch: one per tile */
    int32_t pairs;             /* pairs of x-face boxes whose rows interleave in memory */
    int32_t use_pairs;         /* current tuning: 1 if the batched and per-field forms move those
                                  pairs as contiguous row-boundary segments */
    int32_t staged_mode;       /* current tuning: boxes the batched form loads through tensor maps
                                  (0 none, 1 rows of at most 64 bytes and transposed edges, 2 all
                                  it can) */
    int32_t staged_boxes;      /* boxes the staged kernel takes */
    int32_t staged_items;      /* its work items (one tensor-map load each) */
    int32_t staged_maps;       /* its tensor maps */
    int32_t stages;            /* current tuning: shared-memory stages per staged CTA */
    int32_t stage_bytes;       /* current tuning: bytes per stage */
    int32_t stage_consumers;   /* current tuning: consumer warps per staged CTA */
    int32_t stage_ctas_per_sm; /* current tuning: staged CTAs per SM */
    int32_t gather_scale;      /* current adjoint tuning: gather tiles of short rows halved (-1),
                                  sized by row length (0), doubled (1) or quadrupled (2) */
    int32_t bulk_share;        /* current tuning: quarters (0..4) of the contiguous 16-byte-unit
                                  index-list descriptors that the bulk kernel moves */
    int32_t bulk_tiles;        /* its tiles */
    int32_t gather_bulk;       /* current adjoint tuning: quarters (0..4) of the unstructured owners
                                  whose adjoint the bulk gather kernel takes */
    int32_t gather_bulk_tiles; /* its tiles */
} ghexb_plan_info_t;

/* ---- errors / version ----------------------------------------------------------------- */
int ghexb_last_error(char* buf, size_t len);
int ghexb_version(int* major, int* minor, int* patch);

/* ---- context: replaces ghex::context(MPI_Comm, bool) (context.hpp:20-35, src/context.cpp:14-19).
 * One process owns all domains of the exchange, so no communicator is taken; `device`
 * selects the CUDA device whose memory the fields live in. */
int ghexb_context_create(int device, ghexb_context* out);
int ghexb_context_destroy(ghexb_context ctx);

/* ---- patterns: replace ghex::make_pattern<Grid>(ctx, halo_gen, domains)
 * (pattern_container.hpp:112-146) ------------------------------------------------------ */

/* Regular structured grid: structured::regular::halo_generator(g_first, g_last, halos, periodic)
 * (structured/regular/halo_generator.hpp:68-78) and domain_descriptor(id, first, last)
 * (structured/regular/domain_descriptor.hpp:248-254). dim in 1..3; halos holds 2*dim values
 * (dim0-, dim0+, dim1-, ...); domain_first/last hold n_domains*dim inclusive global coords. */
int ghexb_pattern_create_regular(ghexb_context ctx, int dim, const int* g_first, const int* g_last,
    const int* halos, const int* periodic, int n_domains, const int64_t* domain_ids,
    const int* domain_first, const int* domain_last, ghexb_pattern* out);

/* Staged regular pattern: replaces structured::regular::make_staged_pattern(ctx, domains,
 * domain_lookup, g_first, g_last, halos, periodic) (structured/regular/make_pattern.hpp:47-256).
 * Writes dim patterns to out[0..dim): pattern i exchanges the halos of dimension i over the
 * domain grown by the halos of dimensions 0..i-1, so that exchanging the patterns one after the
 * other fills edges and corners through the faces. neighbor_ids[(d*dim + i)*2 + s] is the id
 * that domain_lookup(id of domain d, offset -1 (s = 0) or +1 (s = 1) along dimension i) returns;
 * it is read only where domain d has a halo on that side. Fails with GHEXB_ERR_INVALID where a
 * receive space has no send space of the same shape feeding it. */
int ghexb_pattern_create_regular_staged(ghexb_context ctx, int dim, const int* g_first, const int* g_last,
    const int* halos, const int* periodic, int n_domains, const int64_t* domain_ids,
    const int* domain_first, const int* domain_last, const int64_t* neighbor_ids, ghexb_pattern* out);

/* Cubed sphere: cubed_sphere::halo_generator(halos) (structured/cubed_sphere/halo_generator.hpp:59-71)
 * and domain_descriptor(cube{edge_size, levels}, tile, x_first, x_last, y_first, y_last)
 * (structured/cubed_sphere/domain_descriptor.hpp:92-104). halos holds 4 values in the order of
 * the reference's m_halo array: [0] -x, [1] +x, [2] -y, [3] +y. Domain ids are (tile, x_first,
 * y_first); ghexb_field_wrap addresses a cubed-sphere domain by its index in this list. */
int ghexb_pattern_create_cubed_sphere(ghexb_context ctx, int edge_size, int levels,
    const int* halos, int n_domains, const int* tiles, const int* x_first, const int* x_last,
    const int* y_first, const int* y_last, ghexb_pattern* out);

/* Unstructured: unstructured::domain_descriptor(id, gids, outer_lids)
 * (unstructured/user_concepts.hpp:145-174) and halo_generator() / halo_generator(gids)
 * (user_concepts.hpp:232-255), pattern set-up of unstructured/pattern.hpp:187-370.
 * Domain k owns gids[gid_offsets[k] .. gid_offsets[k+1]) in storage order and its outer
 * (halo) local ids outer_lids[outer_offsets[k] .. outer_offsets[k+1]). If halo_gid_offsets is
 * NULL every outer gid is a halo (halo_generator()); otherwise domain k's halo is the gid list
 * halo_gids[halo_gid_offsets[k] .. halo_gid_offsets[k+1]) (halo_generator(gids)). */
int ghexb_pattern_create_unstructured(ghexb_context ctx, int n_domains, const int64_t* domain_ids,
    const int64_t* gid_offsets, const int64_t* gids, const int64_t* outer_offsets,
    const int64_t* outer_lids, const int64_t* halo_gid_offsets, const int64_t* halo_gids,
    ghexb_pattern* out);

/* Unstructured with a receive domain ids generator: replaces make_pattern<unstructured::grid>(ctx,
 * halo_gen, recv_domain_ids_gen, domains) (pattern_container.hpp:137-146, unstructured/pattern.hpp:
 * 371-588). Domains and halo generator as above; for domain k, hint_domain_ids and
 * hint_remote_indices [hint_offsets[k] .. hint_offsets[k+1]) give, for each halo element in the
 * halo generator's order, the id of its owner domain and its local index there (the generator's
 * domain_ids() and remote_indices(); ranks are not needed in one process). Receive lists group
 * the halo by owner, send lists hold the remote indices in the receiver's order, tags are
 * (owner id << 7) + receiver id. A remote index must name an inner element of its owner. */
int ghexb_pattern_create_unstructured_hinted(ghexb_context ctx, int n_domains, const int64_t* domain_ids,
    const int64_t* gid_offsets, const int64_t* gids, const int64_t* outer_offsets,
    const int64_t* outer_lids, const int64_t* halo_gid_offsets, const int64_t* halo_gids,
    const int64_t* hint_offsets, const int64_t* hint_domain_ids, const int64_t* hint_remote_indices,
    ghexb_pattern* out);

int ghexb_pattern_destroy(ghexb_pattern p);

/* Introspection, mirroring pattern::recv_halos()/send_halos() (structured/pattern.hpp:184-187). */
int ghexb_pattern_num_domains(ghexb_pattern p, int* n);
int ghexb_pattern_domain_id(ghexb_pattern p, int domain_index, int64_t* id);
int ghexb_pattern_max_tag(ghexb_pattern p, int* max_tag);
/* Number of (neighbour, iteration space) entries received (send==0) or sent (send==1) by a domain. */
int ghexb_pattern_num_spaces(ghexb_pattern p, int domain_index, int send, int* n);
/* Structured entry k: neighbour domain index, local first/last and global first/last, 4 ints each
 * (regular: x,y,z padded with 0; cubed sphere: tile,x,y,z as in the reference). */
int ghexb_pattern_space(ghexb_pattern p, int domain_index, int send, int k, int* neighbor_index,
    int* local_first, int* local_last, int* global_first, int* global_last);
/* Unstructured entry k: neighbour domain index and its local-index list (receiver's halo order). */
int ghexb_pattern_space_indices(ghexb_pattern p, int domain_index, int send, int k,
    int* neighbor_index, int64_t* lids, int64_t capacity, int64_t* count);

/* ---- fields bound to a pattern: replace wrap_field<Arch, Layout>(dom, data, offsets, extents
 * [, strides], device) (structured/regular/field_descriptor.hpp:167-194),
 * cubed_sphere::field_descriptor(dom, data, offsets, extents, ncomp, is_vector)
 * (structured/cubed_sphere/field_descriptor.hpp:113-121) and pattern(field) -> buffer_info
 * (pattern_container.hpp:88-95).
 * ndim: domain dimension, plus one trailing component dimension when num_components > 1
 * (regular) — cubed-sphere fields are always (x, y, z, c).
 * layout_map: ndim ints, gridtools convention (the largest value has stride 1); NULL means
 * x fastest, i.e. {ndim-1, ..., 0}.
 * byte_strides: NULL to derive strides from layout_map and extents (field_utils.hpp:92-111).
 * domain: the domain id (regular) or the domain's index (cubed sphere). */
int ghexb_field_wrap(ghexb_pattern p, int64_t domain, int dtype, void* data, int ndim,
    const int* offsets, const int* extents, const int* layout_map, const int64_t* byte_strides,
    int num_components, int is_vector, ghexb_field* out);

/* Replaces unstructured::data_descriptor<gpu,...>(dom, field, levels, levels_first, outer_stride)
 * (unstructured/user_concepts.hpp:524-535). outer_stride 0 means no padding. */
int ghexb_field_wrap_unstructured(ghexb_pattern p, int64_t domain_id, int dtype, void* data,
    int64_t levels, int levels_first, int64_t outer_stride, ghexb_field* out);

int ghexb_field_destroy(ghexb_field f);

/* ---- host memory for fields (no GHEX counterpart: GHEX exchanges CPU fields on the CPU). A field
 * may live in host memory that the device addresses at the same address: pinned memory
 * (cudaHostAlloc) as it is, ordinary pageable memory after ghexb_host_register, which page-locks
 * [ptr, ptr + bytes) and maps it for the device (cudaHostRegister, mapped and portable). The
 * exchange kernels then read and write such fields in place over the host interconnect. *owned is
 * 1 when the call registered pages of the range (undo with ghexb_host_unregister(ptr)) and 0 when
 * the whole range was page-locked already; pages locked by other code inside the range are left
 * to it, the others registered, and every page is checked. Fails with GHEXB_ERR_INVALID when the
 * device cannot address the memory at its host address. Plans check every page of a host field
 * and refuse memory that the device cannot address, before any launch. */
int ghexb_host_register(void* ptr, size_t bytes, int* owned);
/* *mapped = 1 when every byte of [ptr, ptr + bytes) is device memory, or host memory page-locked
 * and mapped for the device at its own address (pinned allocations, earlier registrations):
 * such a field needs no ghexb_host_register. */
int ghexb_host_is_mapped(const void* ptr, size_t bytes, int* mapped);
/* Page-locked host memory mapped for every device (cudaHostAlloc, mapped and portable), for fields
 * that live in host memory: the device reads and writes it over the host interconnect at its host
 * address. Free with ghexb_host_free. */
int ghexb_host_alloc(size_t bytes, void** out);
int ghexb_host_free(void* ptr);
int ghexb_host_unregister(void* ptr);

/* ---- communication object: replaces make_communication_object<Pattern>(ctx)
 * (communication_object.hpp:653-660), exchange(buffer_info...) (:233-240) and
 * communication_handle::wait/is_ready (:627-640). The exchange of the given fields is ordered on
 * `stream` (NULL = legacy default stream); wait() blocks the host until it has completed,
 * like the reference's wait() (:503-512). A second exchange before wait() fails with
 * GHEXB_ERR_BUSY. Fields of the same pattern are matched across domains by their order in
 * `fields`: the k-th field given for domain a pairs with the k-th field given for domain b. */
int ghexb_co_create(ghexb_context ctx, ghexb_co* out);
int ghexb_co_destroy(ghexb_co co);
int ghexb_co_exchange(
    ghexb_co co, const ghexb_field* fields, int n, void* stream, ghexb_handle* out);
/* Unstructured in-place receive: replaces make_communication_object_ipr(ctx, buffer_info)
 * (unstructured/communication_object_ipr.hpp:188-196) and its exchange() (:146-152). GHEX
 * receives a neighbour's message as raw bytes at the address of the first index of the receive
 * list (:127-141), so the k-th received value lands on halo row first + k. Here the exchange of
 * such a communication object places the values the same way, in one stream-ordered kernel for
 * all given fields; it fails with GHEXB_ERR_INVALID where those rows are not halo rows received
 * once, or where a field's levels are not contiguous rows (levels first, no padding). */
int ghexb_co_create_ipr(ghexb_context ctx, ghexb_co* out);
int ghexb_handle_wait(ghexb_handle h);
int ghexb_handle_is_ready(ghexb_handle h, int* ready);
int ghexb_handle_destroy(ghexb_handle h);

/* ---- explicit plans: the work-descriptor table of one field set, built once and reused.
 * No reference counterpart: GHEX rebuilds its message layout on every exchange
 * (communication_object.hpp:536-624). */
int ghexb_plan_create(ghexb_context ctx, const ghexb_field* fields, int n, ghexb_plan* out);
/* The plan of an in-place receive exchange (see ghexb_co_create_ipr). */
int ghexb_plan_create_ipr(ghexb_context ctx, const ghexb_field* fields, int n, ghexb_plan* out);
int ghexb_plan_destroy(ghexb_plan plan);

/* ---- sharded exchange, one process per GPU: replaces the remote sends and receives of an
 * exchange between ranks (communication_object.hpp:433-512 posting oomph messages,
 * packer.hpp:32-59 packing them). Every process builds the same patterns over all domains;
 * `fields` holds the fields of every domain, those of other processes wrapped around their
 * memory mapped into this one (ghexb_ipc_open), and local[i] != 0 marks this process's own.
 * mode 1 (pull) keeps the descriptors that write a local field: the kernel reads peers'
 * interiors and fills this process's halos. mode 2 (push) keeps those that read a local field:
 * the kernel writes this process's interior values into peers' halos; its adjoint gathers every
 * image of the local owners (the pull form has no adjoint). No descriptor is in two processes'
 * plans, and together they hold every descriptor of the exchange. The caller orders the
 * processes: every process's fields must be final before any process launches, and no process
 * may change its fields until every process's launch is done (a barrier on both sides). The
 * staged form, the bulk column kernel and rebinding are not available on sharded plans. */
int ghexb_plan_create_sharded(ghexb_context ctx, const ghexb_field* fields, int n, const unsigned char* local, int mode,
    ghexb_plan* out);
/* Host-only replay of a sharded plan's tables (as ghexb_plan_check, and every descriptor and
 * adjoint owner checked to be this process's); elements_checked is the number of halo elements
 * its forward kernel writes. */
int ghexb_plan_check_sharded(ghexb_context ctx, const ghexb_field* fields, int n, const unsigned char* local, int mode,
    int64_t* elements_checked);
/* CUDA IPC of field memory (device memory from cudaMalloc, as PyTorch's caching allocator
 * uses): `handle` (64 bytes) names the allocation holding `ptr`, `offset` the byte of `ptr` in
 * it. ghexb_ipc_open maps another process's allocation once per process (later openings of the
 * same handle count references) and returns the address of byte `offset`; ghexb_ipc_close drops
 * one opening. A process cannot open its own handles. */
#define GHEXB_IPC_HANDLE_BYTES 64
int ghexb_ipc_export(const void* ptr, unsigned char* handle, int64_t* offset);
int ghexb_ipc_open(const unsigned char* handle, int64_t offset, void** ptr);
int ghexb_ipc_close(const unsigned char* handle);

/* Host-only validation, no device needed: builds the plan's tables and replays the address
 * computation of every element the forward and adjoint kernels touch, failing with
 * GHEXB_ERR_RANGE if one falls outside its field's memory span. The staged form is replayed in
 * every mode at two stage sizes (its loads inside their tensor maps, every staged box's elements
 * moved once); elements_checked counts the element kernel's form. */
int ghexb_plan_check(ghexb_context ctx, const ghexb_field* fields, int n, int64_t* elements_checked);
int ghexb_plan_get_info(ghexb_plan plan, ghexb_plan_info_t* info);
/* Host-only, no device needed: the least DRAM traffic of one exchange of these fields from a
 * cold cache, with `sector_bytes` (a power of two >= 16) as the DRAM access granularity: every
 * sector holding a halo source element is read, every sector holding a halo element is written
 * back, and a sector written in part that holds no source element is read before it is written.
 * The bytes no kernel can avoid, against which a kernel's measured DRAM traffic is compared. No
 * reference counterpart. */
int ghexb_plan_dram_floor(ghexb_context ctx, const ghexb_field* fields, int n, int sector_bytes, int64_t* read_bytes,
    int64_t* write_bytes);
/* elems_per_thread (4, 8 or 16) and block (a multiple of 32, at most 512); values <= 0 keep the
 * current one. A tile holds elems_per_thread * block elements (half as many 16-byte units).
 * use_pairs: 1 moves the x-face pairs as contiguous segments, 0 as separate boxes, < 0 keeps.
 * Invalidates the captured graph. */
int ghexb_plan_set_tuning(ghexb_plan plan, int elems_per_thread, int block, int use_pairs);
/* Staged form of the batched exchange (no GHEX counterpart): the boxes selected by `mode` (0
 * none, 1 rows of at most 64 bytes and edges whose source rows run along the destination's second
 * axis, 2 every box a tensor map can load) are moved by a second kernel that loads their source
 * regions into shared memory through tensor maps (cp.async.bulk.tensor) and writes the halos from
 * there, beside the element kernel; `stages` (2..16) stages of `stage_bytes` (a multiple of 128)
 * per CTA, `consumers` (1..8) writing warps per CTA, `ctas_per_sm` CTAs per SM. Values <= 0 keep
 * the current one (mode < 0 keeps). Fields in host memory stay on the element kernel.
 * Invalidates the captured graph. */
int ghexb_plan_set_staged(ghexb_plan plan, int mode, int stages, int stage_bytes, int consumers, int ctas_per_sm);
/* Bulk column kernel (no GHEX counterpart): index-list descriptors whose columns are contiguous
 * and in 16-byte units, between device fields, move by the asynchronous copy engine
 * (cp.async.bulk through shared memory) instead of the element kernel: list i when i % 4 < share
 * (0 none, 4 all), beside the element kernel on a second stream when both have work. The batched
 * form only. Invalidates the captured graph. */
int ghexb_plan_set_bulk(ghexb_plan plan, int share);
/* Adjoint tiles (no GHEX counterpart): the gather form's tiles of short rows are sized by row
 * length (gather_scale 0), halved (-1), doubled (1) or quadrupled (2), never beyond a full tile.
 * Invalidates the captured graphs. */
int ghexb_plan_set_adjoint_tuning(ghexb_plan plan, int gather_scale);
/* Bulk form of the unstructured adjoint (no GHEX counterpart): of every owner group whose columns
 * are contiguous and 16-byte aligned, the first `share` quarters (0..4) of the owners are gathered
 * by a kernel that moves their columns with the asynchronous copy engine (cp.async.bulk) through
 * shared memory, beside the element gather kernel on a second stream. The additions keep the
 * receive order: the result is the same bit for bit. Invalidates the captured graphs. */
int ghexb_plan_set_adjoint_bulk(ghexb_plan plan, int share);
/* Status word of the staged and bulk kernels since the last call, then cleared: 0 when every wait
 * ended in time; bit 0 a load (staged or bulk kernel), bit 1 a staged write, bit 2 a bulk gather
 * load that gave up waiting (its halos or owners are then incomplete). Synchronises the device. */
int ghexb_plan_staged_status(ghexb_plan plan, unsigned* status);
/* One forward exchange in the given form, stream-ordered. */
int ghexb_plan_launch(ghexb_plan plan, int form, void* stream);
/* The batched form captured once into a CUDA graph and replayed on `stream`. */
int ghexb_plan_graph_launch(ghexb_plan plan, void* stream);
/* Adjoint of the exchange: every halo value is added into the interior value it was copied
 * from (negated where the forward negated it), in a fixed order, then the halo is zeroed.
 * Float fields only. */
int ghexb_plan_adjoint_launch(ghexb_plan plan, void* stream);
/* Moves a plan to new field memory: data[i] replaces the data pointer of the plan's i-th field
 * (same shape, strides and dtype; the caller guarantees it). The device tables are rewritten on
 * `stream`, ordered with the plan's launches on that stream. Used by the differentiable exchange,
 * whose fields and gradients are new tensors at every step. */
int ghexb_plan_rebind(ghexb_plan plan, void* const* data, int n, void* stream);
/* Times the candidate tunings on `stream` with CUDA events and keeps the fastest one; the
 * chosen tuning is returned through `info` when it is not NULL. Runs real exchanges. Then, for
 * float fields in device memory, times the adjoint's gather-tile sizes (ghexb_plan_set_adjoint_
 * tuning) on the fields, whose memory it saves to a device buffer first and restores after;
 * without room for that copy the adjoint keeps its tiles. */
int ghexb_plan_autotune(ghexb_plan plan, void* stream, int repeats, ghexb_plan_info_t* info);

/* ---- batched exchange without device allocation. This entry point has no counterpart in GHEX.
 * For callers that cannot allocate device memory when they exchange: an application whose memory
 * manager owns the device memory (a pool that reserved HBM at start-up and treats any other
 * cudaMalloc as a failure), or code that must not call cudaMalloc/cudaFree because they may
 * synchronize the device. The work tables go into one fixed device array of 4 MiB that every GPU
 * holds while the library is loaded; exchanges whose tables are larger fail with
 * GHEXB_ERR_RANGE. Each call copies the index lists and forward tiles into the array and
 * launches one batched exchange kernel on `stream` at the default tuning; no cudaMalloc or
 * cudaFree is called. Every call must be made with the context's device current (else
 * GHEXB_ERR_INVALID); the first call on a device also looks up the array's device address. The
 * call cannot be captured into a CUDA graph: a capturing stream is refused with
 * GHEXB_ERR_INVALID. All calls share the array and it keeps the last call's tables: calls that
 * overlap on the GPU race on it. */
int ghexb_exchange_noalloc(ghexb_context ctx, const ghexb_field* fields, int n, void* stream);

/* ---- calibration (no GHEX counterpart): copies `rows` rows of n elements (4 or 8 bytes) at the
 * given element strides, dst[r*dst_stride + i] = src[r*src_stride + i], with the lane mapping of
 * the exchange kernel's box tiles (consecutive threads take consecutive elements, 8 loads in flight
 * per thread) but no work records: the rate at which a plain kernel moves such rows, from device
 * or from mapped host memory, against which the exchange of the same rows is compared. mode 0
 * copies, 1 only reads the source rows, 2 only writes the destination rows. */
int ghexb_calibrate_rows(const void* src, void* dst, int64_t rows, int n, int64_t src_stride, int64_t dst_stride,
    int elem_bytes, int mode, void* stream);

/* ---- the compute step of the differentiable-exchange program. No counterpart in GHEX, which
 * has no stencil: this is the 7-point update x <- x + alpha * L(x) on the interior of each of n
 * 3-D domains (output halo set to 0), or with adjoint != 0 its transpose (gradient of the
 * output's interior in, gradient of the whole input array out). dtype GHEXB_F32 or GHEXB_F64;
 * extents (3 per domain, halo included) and element strides (3 per domain) in x, y, z order;
 * every extent > 2 * halo, halo >= 1; in[i] and out[i] must not overlap. Arithmetic is
 * round-to-nearest in a fixed order without fused multiply-adds. */
int ghexb_stencil7(int dtype, int n, const void* const* in, void* const* out, const int64_t* extents,
                   const int64_t* strides, int halo, double alpha, int adjoint, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GHEX_B200_H */
