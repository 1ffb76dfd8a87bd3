/*
 * viprs_b200.h -- C ABI of the B200 (sm_100a) resample path of viprs.
 *
 * Plain C: pointers, sizes and an opaque stream handle (a cudaStream_t passed
 * as void*, NULL = the legacy default stream).  No entry point aborts or
 * traps; each returns a viprs_status.  Images are row-major, band-interleaved
 * (HWC) like viprs tiles (crates/viprs-core/src/image/region.rs:18-26).
 *
 * Device entry points take device pointers owned by the caller and enqueue
 * work on `stream`; host entry points (suffix _host) copy host buffers in and
 * out inside the call and synchronise the stream before returning.
 *
 * Each entry point names the viprs interface it stands in for.  viprs itself
 * exposes only image handles over its C ABI (src/ffi.rs:58-233,
 * include/viprs.h:1-24); the resample entry points below are what a Rust
 * `DynOperation` bridge (crates/viprs-core/src/op/dynamic_op.rs:16) or the
 * PipelineBuilder methods (crates/viprs-runtime/src/pipeline/builder/
 * resample.rs) would bind to run the op on the GPU.
 */
#ifndef VIPRS_B200_H
#define VIPRS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VIPRS_B200_ABI_VERSION 1

/* Status codes.  Build-time rejections mirror viprs's BuildError variants
   (crates/viprs-core/src/error.rs): InvalidReduceParameters -> INVALID_ARGUMENT,
   tap limit -> TOO_MANY_TAPS, InvalidKernel -> INVALID_KERNEL,
   DegenerateAffineTransform -> DEGENERATE_AFFINE, UnsupportedFormat ->
   UNSUPPORTED_FORMAT. */
typedef enum {
    VIPRS_OK = 0,
    VIPRS_ERR_INVALID_ARGUMENT = 1,
    VIPRS_ERR_UNSUPPORTED_FORMAT = 2,
    VIPRS_ERR_TOO_MANY_TAPS = 3,
    VIPRS_ERR_OUT_OF_MEMORY = 4,
    VIPRS_ERR_CUDA = 5,
    VIPRS_ERR_TIMEOUT = 6,
    VIPRS_ERR_INVALID_KERNEL = 7,
    VIPRS_ERR_DEGENERATE_AFFINE = 8,
    VIPRS_ERR_NULL_POINTER = 9,
    VIPRS_ERR_SIZE_MISMATCH = 10,
    VIPRS_ERR_SCRATCH_LIMIT = 11  /* viprs_reduce_noalloc: tables + planes exceed its static scratch */
} viprs_status;

/* BandFormatId subset on this path (crates/viprs-core/src/format.rs). */
typedef enum { VIPRS_U8 = 0, VIPRS_U16 = 1, VIPRS_F32 = 2 } viprs_format;

/* InterpolationKernel discriminants (crates/viprs-core/src/kernel.rs:22-47). */
typedef enum {
    VIPRS_KERNEL_NEAREST = 0, VIPRS_KERNEL_BILINEAR = 1, VIPRS_KERNEL_BICUBIC = 2,
    VIPRS_KERNEL_QUADRATIC = 3, VIPRS_KERNEL_NOHALO = 4, VIPRS_KERNEL_LBB = 5,
    VIPRS_KERNEL_VSQBS = 6, VIPRS_KERNEL_CATMULLROM = 7, VIPRS_KERNEL_LANCZOS2 = 8,
    VIPRS_KERNEL_LANCZOS3 = 9
} viprs_kernel;

/* ExtendMode (crates/viprs-core/src/shared_ops/extend_mode.rs:5-23). */
typedef enum {
    VIPRS_EXTEND_BLACK = 0, VIPRS_EXTEND_WHITE = 1, VIPRS_EXTEND_BACKGROUND = 2,
    VIPRS_EXTEND_COPY = 3, VIPRS_EXTEND_REPEAT = 4, VIPRS_EXTEND_MIRROR = 5
} viprs_extend;

/* ThumbnailTarget (crates/viprs-ops-spatial/src/resample/thumbnail.rs:116-136). */
typedef enum {
    VIPRS_THUMB_FITBOX = 0, VIPRS_THUMB_FORCE_EXACT = 1, VIPRS_THUMB_WIDTH = 2,
    VIPRS_THUMB_HEIGHT = 3
} viprs_thumb_target;

/* An image buffer.  row_stride is in bytes; 0 means width*bands*sample size.
   data is aligned to the sample size; a nonzero stride is a multiple of the
   sample size and at least that size (else INVALID_ARGUMENT). */
typedef struct {
    void *data;
    uint32_t width;
    uint32_t height;
    uint32_t bands;
    int32_t format;
    uint64_t row_stride;
} viprs_image;

/* ---------------------------------------------------------------- info */
const char *viprs_status_string(int32_t status);
/* Last CUDA error code seen by this thread (0 if none). */
int32_t viprs_last_cuda_error(void);
/* Host evaluation of the sine the device Lanczos2/3 weights use (rounded to
   nearest, |x| <= 2^20; kernel.rs:133-214 calls the platform sin): out[i] =
   sin(x[i]) for i < n.  Returns VIPRS_OK, or INVALID_ARGUMENT for NULL
   pointers with n > 0. */
int32_t viprs_sin_rn(const double *x, double *out, int64_t n);
/* ReduceConfig::output_len (crates/viprs-core/src/resample.rs:92-98). */
uint32_t viprs_reduce_output_len(double factor, uint32_t input_len);
/* Number of filter taps and the 65 x taps fixed-point table of ReduceKernel
   (resample/reduce_common.rs:137-164, 279-316); coeffs may be NULL. */
int32_t viprs_reduce_kernel_table(double factor, int32_t kernel, int32_t *taps,
                                  int16_t *coeffs_i16);

/* ---------------------------------------------------------------- single ops
   Each replaces the viprs op's `process_region` over the whole image
   (the RayonScheduler tile loop, rayon_scheduler/execute.rs:174) for an
   image read from a MemorySource (edge-replicating reads,
   crates/viprs-runtime/src/sources/memory.rs:186-215).  `out` must have the
   op's output size and the input's bands and format. */

/* PipelineBuilder::reduce_h -> ReduceH::process_region (resample/reduceh.rs:100-163). */
int32_t viprs_reduceh(const viprs_image *in, const viprs_image *out, double factor,
                      int32_t kernel, void *stream);
/* PipelineBuilder::reduce_v -> ReduceV::process_region (resample/reducev.rs:99-162). */
int32_t viprs_reducev(const viprs_image *in, const viprs_image *out, double factor,
                      int32_t kernel, void *stream);
/* PipelineBuilder::reduce -> ReduceOp::process_region (resample/reduce.rs:103-251). */
int32_t viprs_reduce(const viprs_image *in, const viprs_image *out, double hfactor,
                     double vfactor, int32_t kernel, void *stream);
/* PipelineBuilder::shrink_h_with_ceil -> ShrinkH::process_region (resample/shrinkh.rs:255-397). */
int32_t viprs_shrinkh(const viprs_image *in, const viprs_image *out, uint32_t factor,
                      int32_t ceil_mode, void *stream);
/* PipelineBuilder::shrink_v_with_ceil -> ShrinkV::process_region (resample/shrinkv.rs:153-236). */
int32_t viprs_shrinkv(const viprs_image *in, const viprs_image *out, uint32_t factor,
                      int32_t ceil_mode, void *stream);
/* PipelineBuilder::shrink -> Shrink::process_region (resample/shrink.rs:179-293). */
int32_t viprs_shrink(const viprs_image *in, const viprs_image *out, uint32_t hfactor,
                     uint32_t vfactor, void *stream);
/* PipelineBuilder::similarity -> SimilarityOp::new_auto_canvas
   (resample/similarity.rs:47-81, 178-232; builder/resample.rs:595-626): scale
   and rotate by `angle` degrees about the origin onto the transformed
   bounding box (libvips's canvas rounding), i.e. an affine with Background(0).
   A scale that is not finite and positive counts as 1.  `out` has the canvas
   size viprs_similarity_node reports. */
int32_t viprs_similarity(const viprs_image *in, const viprs_image *out, double scale, double angle,
                         int32_t kernel, void *stream);
/* PipelineBuilder::zoom -> Zoom::process_region (structural/zoom.rs:310-398;
   builder/geometry.rs:618-643): integer nearest-neighbour upscale, output
   (x, y) = input (x / xfac, y / yfac), output size width*xfac x height*yfac.
   A zero factor is INVALID_ARGUMENT. */
int32_t viprs_zoom(const viprs_image *in, const viprs_image *out, uint32_t xfac, uint32_t yfac,
                   void *stream);
/* PipelineBuilder::premultiply -> Premultiply<U8> (structural/premultiply.rs:84-121). */
int32_t viprs_premultiply(const viprs_image *in, const viprs_image *out, void *stream);
/* PipelineBuilder::unpremultiply -> Unpremultiply<U8|F32> (structural/unpremultiply.rs:76-175). */
int32_t viprs_unpremultiply(const viprs_image *in, const viprs_image *out, void *stream);
/* PipelineBuilder::affine (builder/resample.rs:455-476): FORWARD matrix
   [a,b,c,d] and translation, Background(0) extend, SmallTile tiling. */
int32_t viprs_affine(const viprs_image *in, const viprs_image *out, const double matrix[4],
                     double tx, double ty, int32_t kernel, void *stream);
/* Affine::try_new(..).with_extend().with_source_bounds().with_premultiplied()
   (resample/affine/interpolation.rs:13-40, affine/core.rs:1593-1632) with a
   BACKWARD matrix (output -> input).  tile_w/tile_h give the scheduler tile
   grid whose origins restart the incremental position walk (0 = 128). */
int32_t viprs_affine_backward_matrix(const viprs_image *in, const viprs_image *out,
                                     const double backward[4], double tx, double ty,
                                     int32_t kernel, int32_t extend, double background,
                                     int32_t premultiplied, uint32_t tile_w, uint32_t tile_h,
                                     void *stream);
/* MapImOp (resample/mapim.rs:1135-1274): index is a 2-band f32 image of
   source coordinates with the output's size. */
int32_t viprs_mapim(const viprs_image *src, const viprs_image *index, const viprs_image *out,
                    int32_t kernel, int32_t extend_copy, double background,
                    int32_t premultiplied, void *stream);

/* ---------------------------------------------------------------- chains
   One node per PipelineBuilder method call on this path (builder/resample.rs);
   kinds follow ThumbnailNode / ResizeNode (thumbnail.rs:42-104) plus Reduce and
   Shrink.  Affine nodes carry the BACKWARD matrix (output -> input), as
   PipelineBuilder::affine stores it after forward_affine_to_backward. */
typedef enum {
    VIPRS_NODE_PREMULTIPLY = 1, VIPRS_NODE_SHRINKH = 2, VIPRS_NODE_SHRINKV = 3,
    VIPRS_NODE_REDUCEH = 4, VIPRS_NODE_REDUCEV = 5, VIPRS_NODE_AFFINE = 6,
    VIPRS_NODE_EXTRACT_AREA = 7, VIPRS_NODE_UNPREMULTIPLY = 8,
    VIPRS_NODE_ZOOM = 9,    /* factors in factor_u (x) / vfactor_u (y) */
    VIPRS_NODE_REDUCE = 10, VIPRS_NODE_SHRINK = 11
} viprs_node_kind;

/* DemandHint (crates/viprs-core/src/op/demand.rs:14-27). */
typedef enum {
    VIPRS_DEMAND_ANY = 0, VIPRS_DEMAND_THIN_STRIP = 1, VIPRS_DEMAND_FAT_STRIP = 2,
    VIPRS_DEMAND_SMALL_TILE = 3, VIPRS_DEMAND_FULL_IMAGE = 4, VIPRS_DEMAND_ONE_LINE = 5
} viprs_demand;

typedef struct {
    int32_t kind;
    uint32_t factor_u;      /* shrink factor (horizontal for SHRINK) */
    uint32_t vfactor_u;     /* SHRINK vertical factor */
    int32_t ceil_mode;      /* shrink_h_with_ceil / shrink_v_with_ceil */
    double factor;          /* reduce factor (horizontal for REDUCE) */
    double vfactor;         /* REDUCE vertical factor */
    int32_t kernel;
    double matrix[4];       /* AFFINE backward matrix */
    double tx, ty;
    uint32_t out_width, out_height;
    int32_t extend;
    double background;
    int32_t premultiplied;
    uint32_t area_x, area_y, area_width, area_height;  /* EXTRACT_AREA */
    int32_t demand_hint;    /* the node bridge's DemandHint */
} viprs_node;

/* PipelineBuilder::forward_affine_to_backward (builder/resample.rs:25-60). */
int32_t viprs_forward_affine_to_backward(const double forward[4], double tx, double ty,
                                         double backward[4], double *btx, double *bty);

/* ---------------------------------------------------------------- plans
   A plan is an immutable, device-resident execution of a builder chain:
   coefficient and position tables plus the workspace for intermediates are
   allocated at creation, so execution allocates nothing.  Concurrent
   executions of one plan must not overlap (they share its workspace). */
typedef struct viprs_plan viprs_plan;

/* PipelineBuilder::thumbnail(Thumbnail::new(target, kernel).with_crop(crop))
   over an in-memory source (builder/resample.rs:871-979, thumbnail.rs:204-524). */
int32_t viprs_thumbnail_plan_create(uint32_t width, uint32_t height, uint32_t bands,
                                    int32_t format, int32_t target, uint32_t target_width,
                                    uint32_t target_height, int32_t kernel, int32_t crop,
                                    viprs_plan **out_plan);
/* Thumbnail::into_pipeline_nodes / into_pipeline_nodes_without_shrink_hint
   (thumbnail.rs:204-524), host only: the planned nodes (kind 9 = the Zoom
   upscale), the output size and the shrink-on-load hint (0 = none).  Returns
   SIZE_MISMATCH, with *n_nodes set, when `capacity` nodes do not suffice. */
int32_t viprs_thumbnail_plan_nodes(int32_t target, uint32_t target_width, uint32_t target_height,
                                   int32_t kernel, int32_t crop, uint32_t width, uint32_t height,
                                   uint32_t bands, int32_t allow_shrink_hint, viprs_node *nodes,
                                   int32_t capacity, int32_t *n_nodes, uint32_t *out_width,
                                   uint32_t *out_height, uint32_t *shrink_factor);
/* Resize::with_gap(gap).into_pipeline_nodes (resize.rs:89-348), host only:
   the planned nodes (kind 9 = the Zoom upscale, its factors in factor_u /
   vfactor_u) and the output size.  SIZE_MISMATCH, with *n_nodes set, when
   `capacity` nodes do not suffice. */
int32_t viprs_resize_plan_nodes(double hscale, double vscale, int32_t kernel, double gap,
                                uint32_t width, uint32_t height, viprs_node *nodes,
                                int32_t capacity, int32_t *n_nodes, uint32_t *out_width,
                                uint32_t *out_height);
/* Host only: the output size of a node chain on a width x height source
   (PipelineBuilder::current_dimensions after those builder calls). */
int32_t viprs_chain_output_size(uint32_t width, uint32_t height, const viprs_node *nodes,
                                int32_t n_nodes, uint32_t *out_width, uint32_t *out_height);
/* Host only: the Affine node PipelineBuilder::similarity runs on a width x
   height image (backward matrix, canvas translation in tx / ty, canvas size in
   out_width / out_height, SmallTile hint), for a chain plan or a batch. */
int32_t viprs_similarity_node(double scale, double angle, int32_t kernel, uint32_t width,
                              uint32_t height, viprs_node *node);
/* PipelineBuilder::resize(Resize::new(hscale, vscale, kernel)) (builder/resample.rs:637-711). */
int32_t viprs_resize_plan_create(uint32_t width, uint32_t height, uint32_t bands, int32_t format,
                                 double hscale, double vscale, int32_t kernel,
                                 viprs_plan **out_plan);
/* PipelineBuilder::from_source(MemorySource)...build() for an arbitrary node
   chain; demand_override < 0 takes the maximum hint over the nodes
   (pipeline/arena.rs:411-420). */
int32_t viprs_chain_plan_create(uint32_t width, uint32_t height, uint32_t bands, int32_t format,
                                const viprs_node *nodes, int32_t n_nodes, int32_t demand_override,
                                viprs_plan **out_plan);
int32_t viprs_plan_output_size(const viprs_plan *plan, uint32_t *width, uint32_t *height);
/* Synchronise `stream`, then return and clear the plan's device error word:
   VIPRS_OK, or VIPRS_ERR_TIMEOUT when a kernel's bounded wait for its bulk
   copies gave up since the last call (its output is then incomplete). */
int32_t viprs_plan_status(viprs_plan *plan, void *stream);
int32_t viprs_plan_workspace_bytes(const viprs_plan *plan, uint64_t *bytes);
/* Number of kernel launches one execution enqueues. */
int32_t viprs_plan_launch_count(const viprs_plan *plan, int32_t *launches);
/* Run the plan on packed device buffers (input and output sizes fixed at creation). */
int32_t viprs_plan_execute(viprs_plan *plan, const void *src, void *dst, void *stream);
/* Run stages [first, first + count) of the plan only (for per-kernel timing;
   stages must be run in order for a full result). */
int32_t viprs_plan_execute_stages(viprs_plan *plan, int32_t first, int32_t count, const void *src,
                                  void *dst, void *stream);
/* Same through host buffers: copy in, run, copy out, synchronise. */
int32_t viprs_plan_execute_host(viprs_plan *plan, const void *host_src, void *host_dst,
                                void *stream);
void viprs_plan_destroy(viprs_plan *plan);

/* ---------------------------------------------------------------- batches
   Thumbnails of many images of uneven size and band count.  No viprs entry
   point corresponds: viprs runs one pipeline per image
   (ImageApi::thumbnail, image_api/transform.rs:287-301); the per-image path
   below is exactly that, one plan per image, and the persistent path runs
   the same plans' stages as a few persistent launches over a device work
   list: one per stage level and kind (the shrinks of every image, then the
   fused reduces, ...), so that launch order carries every dependency. */
typedef struct viprs_batch viprs_batch;

/* One PipelineBuilder::thumbnail plan per image (u8 images). */
int32_t viprs_thumbnail_batch_create(int32_t n_images, const uint32_t *widths,
                                     const uint32_t *heights, const uint32_t *bands,
                                     int32_t target, uint32_t target_width,
                                     uint32_t target_height, int32_t kernel, int32_t crop,
                                     viprs_batch **out_batch);
/* The same node chain (as viprs_chain_plan_create) on every image of the batch
   (u8 images): e.g. reduce_h + reduce_v over many photos of uneven size. */
int32_t viprs_chain_batch_create(int32_t n_images, const uint32_t *widths, const uint32_t *heights,
                                 const uint32_t *bands, const viprs_node *nodes, int32_t n_nodes,
                                 int32_t demand_override, viprs_batch **out_batch);
int32_t viprs_batch_output_size(const viprs_batch *batch, int32_t index, uint32_t *width,
                                uint32_t *height);
/* Work items, stages and the largest persistent grid of the current configuration. */
int32_t viprs_batch_work_items(const viprs_batch *batch, int32_t *items, int32_t *stages,
                               int32_t *grid);
/* Launches per execution: the persistent launches, and the plans' stage count for per-image. */
int32_t viprs_batch_launch_count(const viprs_batch *batch, int32_t *batched, int32_t *per_image);
/* Persistent path.  d_srcs / d_dsts are DEVICE arrays of n_images device
   pointers (packed HWC u8 buffers, 16-byte aligned for the bulk-copy path). */
int32_t viprs_batch_execute(viprs_batch *batch, const uint64_t *d_srcs, const uint64_t *d_dsts,
                            void *stream);
/* The same, through a CUDA graph captured on first use for these arrays. */
int32_t viprs_batch_execute_graph(viprs_batch *batch, const uint64_t *d_srcs,
                                  const uint64_t *d_dsts, void *stream);
/* Plain per-image path: h_srcs / h_dsts are HOST arrays of device pointers. */
int32_t viprs_batch_execute_per_image(viprs_batch *batch, const uint64_t *h_srcs,
                                      const uint64_t *h_dsts, void *stream);
/* Autotuner: times candidate warp-shrink stage budgets (1536, 2048, 3072,
   4096 bytes) x blocks per SM (occupancy maximum, 2, 3) on the given images
   and keeps the fastest. */
int32_t viprs_batch_autotune(viprs_batch *batch, const uint64_t *d_srcs, const uint64_t *d_dsts,
                             void *stream, int32_t repeats, float *best_ms);
/* ring_bytes: the warp shrink's stage budget, the most source bytes one row
   segment of a shrink item may take (1024..32768; each warp holds four such
   stages); ring_slots: kept for the interface, 0..16, no effect on the warp
   shrink; blocks_per_sm: cap of the persistent launches (0 = occupancy
   maximum). */
int32_t viprs_batch_set_config(viprs_batch *batch, uint32_t ring_bytes, int32_t ring_slots,
                               int32_t blocks_per_sm);
int32_t viprs_batch_get_config(const viprs_batch *batch, uint32_t *ring_bytes,
                               int32_t *ring_slots, int32_t *blocks_per_sm);
/* Synchronise `stream` and return the first device-side error (VIPRS_ERR_TIMEOUT
   if a bounded wait gave up), 0 if none. */
int32_t viprs_batch_status(viprs_batch *batch, void *stream);
void viprs_batch_destroy(viprs_batch *batch);

/* ---- no device allocation ----------------------------------------------------
   No counterpart in the reference: viprs runs on the CPU and has no device
   memory to manage.  Same operation, arguments and result as viprs_reduce,
   but the call allocates no device memory (no cudaMalloc, cudaMallocAsync or
   cudaFree, no library allocator): its coefficient and position tables, and
   the intermediate plane when the fused tile does not fit in shared memory,
   live in one static device array of VIPRS_NOALLOC_SCRATCH_BYTES that every
   GPU loading this library holds until the process exits.  It is for callers
   that cannot allocate device memory: a host framework whose allocator owns
   the GPU's memory, a plugin inside another program's processing callback,
   a latency-bound loop that must not let cudaMalloc/cudaFree synchronise the
   device.  Work needing more than the array returns VIPRS_ERR_SCRATCH_LIMIT
   before touching the GPU.  The first call on each device (with that device
   current) looks up the array's device address and may load this library's
   device code there.  All calls on a device share the array, so calls whose
   GPU work overlaps (different streams or threads without ordering between
   them) race; order them. */
#define VIPRS_NOALLOC_SCRATCH_BYTES (4u << 20)
int32_t viprs_reduce_noalloc(const viprs_image *in, const viprs_image *out, double hfactor,
                             double vfactor, int32_t kernel, void *stream);

/* ---- adjoints (backward passes), f32 images ---------------------------------
   viprs's resample operators are forward only, so these have no reference
   counterpart; each is the exact transpose / derivative of the forward entry
   point named beside it, as this library evaluates it (same coefficient
   tables, positions and extend rules; the per-pixel derivative arithmetic is
   f32, positions and matrix sums f64).  Scratch is allocated stream-ordered on
   `stream` from a memory pool the library keeps per device (its memory stays
   mapped between calls).  The reduce adjoints keep each geometry's transposed
   tables on the device after the first call for it, which uploads them with a
   synchronous copy.  Gradients are overwritten, not accumulated. */

/* Transpose of viprs_reduceh (horizontal != 0) / viprs_reducev on f32: for
   every input sample, a gather over the outputs whose taps read it; taps that
   the clamp-to-edge source read folds onto sample 0 / n-1 are folded there. */
int32_t viprs_reduce_adjoint(const viprs_image *grad_out, const viprs_image *grad_in,
                             double factor, int32_t kernel, int32_t horizontal, void *stream);
/* Transpose of the ReduceH -> ReduceV chain (PipelineBuilder::reduce_h(..)
   .reduce_v(..), one fused stage of a chain plan): V^T into a mid plane, then
   H^T folding the mid rows that lie beyond the image onto its edge rows. */
int32_t viprs_reduce_hv_adjoint(const viprs_image *grad_out, const viprs_image *grad_in,
                                double hfactor, double vfactor, int32_t kernel, void *stream);
/* Gradient of viprs_affine_backward_matrix (bilinear) wrt its input image
   (grad_in, may be NULL; f32 atomics, or with `deterministic` a fixed-point
   2^-32 accumulator whose integer adds make the result independent of order)
   and wrt the backward matrix and translation (grad_matrix[6] =
   d/d(b0, b1, b2, b3, tx, ty), DEVICE memory, may be NULL; written on
   `stream` by a fixed-order reduction of per-block partial sums).  4-band
   images without `premultiplied` take the alpha-premultiplying sampler's
   derivative. */
int32_t viprs_affine_grad(const viprs_image *in, const viprs_image *grad_out,
                          const viprs_image *grad_in, const double backward[4], double tx,
                          double ty, int32_t kernel, int32_t extend, double background,
                          int32_t premultiplied, uint32_t tile_w, uint32_t tile_h,
                          int32_t deterministic, double *grad_matrix, void *stream);
/* Gradient of viprs_mapim on f32 wrt the source image (grad_src, scatter as in
   viprs_affine_grad) and wrt the 2-band coordinates (grad_index: derivative of
   the interpolation weights, with the quotient rule through their
   renormalisation); either output may be NULL.  2/4-band sources need
   `premultiplied` (the alpha-premultiplying sampler is forward only). */
int32_t viprs_mapim_grad(const viprs_image *src, const viprs_image *index,
                         const viprs_image *grad_out, const viprs_image *grad_src,
                         const viprs_image *grad_index, int32_t kernel, int32_t extend_copy,
                         double background, int32_t premultiplied, int32_t deterministic,
                         void *stream);

#ifdef __cplusplus
}
#endif
#endif
