/*
 * viprs_oracle.h -- CPU restatement of viprs's resample path, used ONLY as a
 * test oracle and as the timed CPU baseline ("port" kind).
 *
 * This is test infrastructure.  Nothing in the product library links it; the
 * parity tests, the smoke check and the CPU-baseline leg of the bench load it
 * through ctypes to check or time the CUDA path.
 *
 * Every function restates the reference algorithm in plain C with the same
 * floating-point operation order (compiled with -ffp-contract=off so that no
 * multiply-add is fused unless the reference fuses it with `mul_add`).  The
 * citations name files of the viprs 0.1.5 source tree.
 *
 * Parity pin: the restatement is checked against the exact (diff 0) libvips
 * fixtures that viprs's own tests match (tests/fixtures/{reduceh_libvips,
 * reducev_libvips, reduce_libvips, shrink_libvips, libvips_parity_resample,
 * resize_libvips, shrinkh, shrinkv}) and against the known-answer unit tests
 * (reduceh.rs, reduce_common.rs, sample_conv.rs, shrinkv.rs, thumbnail.rs).
 */
#ifndef VIPRS_ORACLE_H
#define VIPRS_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* InterpolationKernel discriminants (crates/viprs-core/src/kernel.rs:22-47). */
enum {
    OR_K_NEAREST = 0, OR_K_BILINEAR = 1, OR_K_BICUBIC = 2, OR_K_QUADRATIC = 3,
    OR_K_NOHALO = 4, OR_K_LBB = 5, OR_K_VSQBS = 6, OR_K_CATMULLROM = 7,
    OR_K_LANCZOS2 = 8, OR_K_LANCZOS3 = 9
};

/* Sample formats handled on this path. */
enum { OR_U8 = 0, OR_U16 = 1, OR_F32 = 2 };

/* DemandHint (crates/viprs-core/src/op/demand.rs:14-27). */
enum { OR_DH_ANY = 0, OR_DH_THIN = 1, OR_DH_FAT = 2, OR_DH_SMALLTILE = 3,
       OR_DH_FULL = 4, OR_DH_ONELINE = 5 };

/* ExtendMode (crates/viprs-core/src/shared_ops/extend_mode.rs:5-23). */
enum { OR_EXT_BLACK = 0, OR_EXT_WHITE = 1, OR_EXT_BACKGROUND = 2, OR_EXT_COPY = 3,
       OR_EXT_REPEAT = 4, OR_EXT_MIRROR = 5 };

/* Op kinds of the restated pipeline. */
enum { OR_OP_SHRINKH = 1, OR_OP_SHRINKV = 2, OR_OP_REDUCEH = 3, OR_OP_REDUCEV = 4,
       OR_OP_REDUCE = 5, OR_OP_PREMULTIPLY = 6, OR_OP_UNPREMULTIPLY = 7,
       OR_OP_AFFINE = 8, OR_OP_SHRINK = 9, OR_OP_EXTRACT = 10,
       OR_OP_ZOOM = 11 /* ufactor = x factor, ceil_mode = y factor */ };

/* Status codes. */
enum { OR_OK = 0, OR_EINVAL = 1, OR_ETAPS = 2, OR_ENOMEM = 3, OR_EFORMAT = 4 };

/* One pipeline node, as materialised by PipelineBuilder. */
typedef struct {
    int32_t kind;
    uint32_t ufactor;      /* shrink factor */
    int32_t ceil_mode;     /* shrink ceil mode */
    double factor;         /* reduce factor (h for REDUCE) */
    double vfactor;        /* REDUCE v factor */
    int32_t kernel;
    int32_t demand_hint;
    /* affine: backward matrix (output -> input), translation, output size */
    double m[4];
    double tx, ty;
    uint32_t out_w, out_h;
    int32_t extend;
    double background;
    int32_t premultiplied;
    /* extract area */
    uint32_t ex, ey, ew, eh;
} or_node;

/* Thumbnail / resize plan node kinds (thumbnail.rs:42-104, resize.rs ResizeNode). */
enum { OR_TN_PREMULTIPLY = 1, OR_TN_SHRINKH = 2, OR_TN_SHRINKV = 3, OR_TN_REDUCEH = 4,
       OR_TN_REDUCEV = 5, OR_TN_AFFINE = 6, OR_TN_EXTRACT = 7, OR_TN_UNPREMULTIPLY = 8,
       OR_TN_ZOOM = 9 };

typedef struct {
    int32_t kind;
    uint32_t ufactor;
    double factor;
    int32_t kernel;
    double m[4];
    double tx, ty;
    uint32_t out_w, out_h;
    uint32_t ex, ey, ew, eh;
    uint32_t zx, zy;
} or_plan_node;

/* ThumbnailTarget (thumbnail.rs:116-136). */
enum { OR_TT_FITBOX = 0, OR_TT_FORCE = 1, OR_TT_WIDTH = 2, OR_TT_HEIGHT = 3 };

/* ---- 1-D kernel weights and reduce tables ---- */
double or_kernel_weight(int32_t kernel, double x);
double or_kernel_support(int32_t kernel);
/* taps/pad_before/offset and the 65-phase tables; returns status. */
int32_t or_reduce_tables(double factor, int32_t kernel, uint32_t input_len, int32_t bind,
                         int32_t *taps, int64_t *pad_before, double *offset,
                         double *coeffs_f64 /* 65*taps or NULL */,
                         int16_t *coeffs_i16 /* 65*taps or NULL */);
/* (start, phase) for a source position. */
void or_reduce_plan(double factor, int32_t kernel, uint32_t input_len, int32_t bind,
                    double index, int64_t *start, int32_t *phase, double *position);

/* ---- planners ---- */
int32_t or_thumbnail_plan(int32_t target, uint32_t tw, uint32_t th, int32_t kernel,
                          int32_t crop, uint32_t in_w, uint32_t in_h, uint32_t bands,
                          int32_t allow_shrink_hint, or_plan_node *nodes, int32_t max_nodes,
                          int32_t *n_nodes, uint32_t *out_w, uint32_t *out_h,
                          uint32_t *shrink_on_load);
int32_t or_resize_plan(double hscale, double vscale, int32_t kernel, double gap,
                       uint32_t in_w, uint32_t in_h, or_plan_node *nodes, int32_t max_nodes,
                       int32_t *n_nodes, uint32_t *out_w, uint32_t *out_h);

/* ---- pipeline execution (MemorySource -> nodes -> MemorySink) ---- */
/* Output dimensions of a node chain. */
int32_t or_pipeline_dims(const or_node *nodes, int32_t n, uint32_t w, uint32_t h,
                         uint32_t *out_w, uint32_t *out_h);
/* Run the chain tile by tile as RayonScheduler does.  demand_override < 0
   means "max over nodes".  threads <= 0 means 1. */
int32_t or_pipeline_run(const void *src, uint32_t w, uint32_t h, uint32_t bands,
                        int32_t fmt, const or_node *nodes, int32_t n,
                        int32_t demand_override, int32_t threads, void *dst,
                        uint32_t out_w, uint32_t out_h);

/* Builder-level conveniences that materialise nodes exactly like
   PipelineBuilder::{thumbnail, resize} (builder/resample.rs:637-711, 871-979). */
int32_t or_thumbnail_run(const void *src, uint32_t w, uint32_t h, uint32_t bands,
                         int32_t fmt, int32_t target, uint32_t tw, uint32_t th,
                         int32_t kernel, int32_t crop, int32_t threads, void *dst,
                         uint32_t *out_w, uint32_t *out_h);
int32_t or_thumbnail_dims(uint32_t w, uint32_t h, uint32_t bands, int32_t target,
                          uint32_t tw, uint32_t th, int32_t kernel, int32_t crop,
                          uint32_t *out_w, uint32_t *out_h);
int32_t or_resize_run(const void *src, uint32_t w, uint32_t h, uint32_t bands,
                      int32_t fmt, double hscale, double vscale, int32_t kernel,
                      int32_t threads, void *dst, uint32_t *out_w, uint32_t *out_h);

/* ---- mapim (mapim.rs:1135-1274), full-image form ----
   index: 2-band image of index_fmt (OR_U8 / OR_U16 / OR_F32), read as f64.
   2/4-band sources with premultiplied == 0 take the alpha-premultiplying
   sampler (mapim.rs:993-1040). */
int32_t or_mapim_run(const void *src, uint32_t sw, uint32_t sh, uint32_t bands, int32_t fmt,
                     const void *index, int32_t index_fmt, uint32_t iw, uint32_t ih, int32_t kernel,
                     int32_t extend_copy, double background, int32_t premultiplied,
                     int32_t threads, void *dst);

#ifdef __cplusplus
}
#endif
#endif
