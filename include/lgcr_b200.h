/*
 * lgcr_b200.h — C ABI of the B200-native LGCR Recon implementation.
 *
 * This is the drop-in boundary for the `lgcr.Recon` path of
 * MysteryDove/vapoursynth-LGCR and its Sharpen, TRecon and Downsample
 * filters.  Every entry point takes plain pointers,
 * sizes and strides; no CUDA, VapourSynth or torch types appear in the
 * signatures (a CUDA stream is passed as `void *`).
 *
 * Reference interfaces replaced (paths are within the reference project):
 *   lgcr_recon_create      <- lgcrCreate            src/plugin.cpp:998-1158
 *   lgcr_recon_destroy     <- lgcrFree              src/plugin.cpp:992-996
 *   lgcr_recon_output_format <- viOut query         src/plugin.cpp:1144-1152
 *   lgcr_recon_frame       <- lgcrGetFrame          src/plugin.cpp:177-721
 *   lgcr_batch_*           <- frame-parallel getFrame calls (fmParallel,
 *                             src/plugin.cpp:1157) folded into one launch
 *   lgcr_sharpen_*         <- sharpenCreate / sharpenGetFrame / sharpenFree
 *                             src/plugin.cpp:14-111
 *   lgcr_trecon_*          <- tReconCreate / tReconGetFrame
 *                             src/plugin.cpp:723-990
 *   lgcr_downsample_*      <- downsampleCreate / downsampleGetFrame /
 *                             downsampleFree src/downsample.cpp:740-918
 *   lgcr_server_*          <- the VapourSynth core's concurrent request
 *                             scheduling of Recon frames (no single
 *                             reference symbol; see plugin.cpp:215-217
 *                             for the per-worker workspace pool it sizes)
 *
 * Status codes are returned, never traps; error strings mirror the
 * reference's mapSetError messages where one exists.
 */
#ifndef LGCR_B200_H
#define LGCR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LGCR_B200_VERSION_MAJOR 2
#define LGCR_B200_VERSION_MINOR 1

/* "argument not given" sentinels (VapourSynth optional arguments) */
#define LGCR_UNSET_INT (-2147483647 - 1)
/* doubles: any NaN means "not given" */

/* status codes */
enum lgcr_status {
    LGCR_OK = 0,
    LGCR_E_INVALID = 1,      /* invalid parameter / format (create-time)   */
    LGCR_E_ARGUMENT = 2,     /* invalid call argument (planes, sizes)      */
    LGCR_E_CUDA = 3,         /* CUDA runtime error                          */
    LGCR_E_NOMEM = 4,        /* device or host allocation failed            */
    LGCR_E_TIMEOUT = 5,      /* bounded wait expired                        */
    LGCR_E_BUSY = 6,         /* admission refused (budget / queue full)     */
    LGCR_E_CLOSED = 7,       /* server shut down                            */
    LGCR_E_INTERNAL = 8
};

/* colour family values follow VapourSynth API v4 numbering */
enum { LGCR_CF_GRAY = 1, LGCR_CF_RGB = 2, LGCR_CF_YUV = 3 };
enum { LGCR_ST_INTEGER = 0, LGCR_ST_FLOAT = 1 };
/* where frame planes live */
enum { LGCR_MEM_HOST = 0, LGCR_MEM_DEVICE = 1 };

/* Input clip format (VSVideoInfo subset used by lgcrCreate). */
typedef struct lgcr_format {
    int color_family;      /* LGCR_CF_*                                   */
    int sample_type;       /* LGCR_ST_*                                   */
    int bits_per_sample;   /* 8..16 integer, 32 float                     */
    int subsampling_w;     /* log2 horizontal chroma subsampling          */
    int subsampling_h;     /* log2 vertical chroma subsampling            */
    int width, height;     /* constant luma dimensions (0 = variable)     */
} lgcr_format;

/*
 * Recon arguments, one field per entry of the reference signature
 *   clip:vnode;width:int:opt;height:int:opt;kernel:data:opt;taps:int:opt;
 *   algo:int:opt;b:float:opt;c:float:opt;strength:float:opt;sigma:float:opt;
 *   sratio:float:opt;sdb:float:opt;stretch:float:opt;gsigma:float:opt;
 *   rescue:float:opt;ridge:int:opt;cedge:int:opt;ar:float:opt;reg:float:opt;
 *   loc:data:opt;sparse:int:opt;bp:float:opt;ms:float:opt;qgate:float:opt;
 *   bm:int:opt                                   (src/plugin.cpp:1166-1171)
 * Ints use LGCR_UNSET_INT, doubles NaN and strings NULL for "not given";
 * lgcr_params_init() sets every field to "not given".
 */
typedef struct lgcr_params {
    int width, height;
    const char *kernel;
    int taps;
    int algo;
    double b, c;
    double strength, sigma, sratio, sdb, stretch, gsigma, rescue;
    int ridge, cedge;
    double ar, reg;
    const char *loc;
    int sparse;
    double bp, ms, qgate;
    int bm;
} lgcr_params;

/* One plane: pointer, row stride in bytes, dimensions in samples. */
typedef struct lgcr_plane {
    void *data;
    ptrdiff_t stride;
    int width, height;
} lgcr_plane;

/* Per-frame work counters (the reference's _LGCR_* profile props,
 * src/plugin.cpp:126-155). Filled only when requested. */
typedef struct lgcr_frame_stats {
    uint64_t output_pixels;
    uint64_t sparse_active_pixels;   /* trust-mask pixels set            */
    uint64_t sparse_total_pixels;
    uint64_t active_output_pixels;   /* guided output pixels             */
    uint64_t active_chroma_pixels;
    double sparse_active_ratio;
    double device_ms;                /* device time of the frame          */
} lgcr_frame_stats;

typedef struct lgcr_recon lgcr_recon;

void lgcr_params_init(lgcr_params *params);

/* lgcrCreate: validate parameters against the clip format and build the
 * filter (host weight tables, jinc LUT, device-resident copies).
 * On failure returns LGCR_E_INVALID and copies the reference's message
 * into err (if err != NULL). */
int lgcr_recon_create(const lgcr_params *params, const lgcr_format *fmt,
                      lgcr_recon **out, char *err, size_t errlen);

/* lgcrFree */
void lgcr_recon_destroy(lgcr_recon *filter);

/* Output clip format: 4:4:4, same sample type and depth, output size. */
int lgcr_recon_output_format(const lgcr_recon *filter, lgcr_format *out);

/*
 * lgcrGetFrame for one frame.
 *   in[0..2]   Y, U, V source planes (format of create())
 *   out[0..2]  Y, U, V output planes (4:4:4, output size). When the output
 *              size equals the input size, out[0].data may be NULL: the
 *              luma plane is then shared with the input and not written
 *              (the reference attaches the source luma by reference,
 *              src/plugin.cpp:265-269).
 *   chroma_location  the frame's _ChromaLocation (0..5), or -1 if absent.
 *   memory     LGCR_MEM_HOST: planes are host memory; the call uploads,
 *              runs and downloads, and returns when the output is written.
 *              LGCR_MEM_DEVICE: planes are device memory; work is enqueued
 *              on `stream` (a cudaStream_t, NULL = legacy default stream)
 *              and the call returns without waiting.
 *   stats      optional; when non-NULL the call waits for the frame and
 *              fills the counters.
 * Safe to call concurrently from several host threads on one filter. */
int lgcr_recon_frame(lgcr_recon *filter, const lgcr_plane in[3],
                     const lgcr_plane out[3], int chroma_location,
                     int memory, void *stream, lgcr_frame_stats *stats);

/* Text of the last error raised on the calling thread. */
const char *lgcr_last_error(void);

/*
 * lgcr_recon_frame_static: lgcr_recon_frame for device planes that
 * allocates no device memory. No counterpart in the reference (which runs on
 * the CPU); it exists for callers that cannot call cudaMalloc -- hosts that
 * own all device memory through their own pool, or latency-critical paths
 * where an allocation would synchronize the device.
 * Scratch lives in one library-wide device array of 64 MiB (held on every
 * GPU that loads the library until exit): frames needing more, and algo 4/6
 * with strength > 0, bm or bp, are rejected with LGCR_E_ARGUMENT and a
 * message. The first call on a device looks up the array's address and
 * should come before any stream capture. All calls share the array: calls
 * whose work overlaps on the GPU race and must be ordered by the caller.
 * Work is enqueued on `stream` (a cudaStream_t) and the call does not wait
 * for the GPU to run it; its uploads of the geometry tables and the frame
 * descriptor read pageable host memory, so the call may block the host until
 * those few kilobytes are staged. A call on a stream that is being captured
 * into a CUDA graph returns LGCR_E_ARGUMENT (the copies would read host
 * memory the call has released).
 */
int lgcr_recon_frame_static(lgcr_recon *filter, const lgcr_plane in[3],
                            const lgcr_plane out[3], int chroma_location, void *stream);

/* Diagnostics: the host-built chroma sampling axis the kernels index
 * (buildChromaAxisUncached, src/kernels.cpp:337-404) for axis 0 (x) or 1
 * (y) at siting `shift`. Arrays hold n entries (n*sup for w/am); any may be
 * NULL. Returns the support in *sup. */
int lgcr_debug_axis(const lgcr_recon *filter, int axis, double shift, int *start,
                    float *w, uint8_t *am, float *pos, float *lpos, int *chroma_i0,
                    float *chroma_f, int *luma_i0, float *luma_f, int *sup);

/* Self-check of the device reciprocal the guided taps use for their
 * 1/(1 + ...) similarity and bump terms (src/recon.cpp:615-619 divides):
 * compares it with the IEEE quotient 1.0f/x for every float x in [1, 2^64)
 * plus the special arguments, on the current device. Writes the number of
 * differing results to *mismatches (0 expected). No counterpart in the
 * reference (its divides are plain C++). */
int lgcr_selftest_reciprocal(uint64_t *mismatches);

/* ---------------------------------------------------------------------
 * Sharpen: the reference's second filter, a 5x5 gated bilateral unsharp
 * mask (luma self-guided; subsampled chroma guided by the sharpened luma's
 * footprint map; 4:4:4 chroma self-guided). Same format in and out.
 *   lgcr_sharpen_create   <- sharpenCreate    src/plugin.cpp:84-111
 *   lgcr_sharpen_frame    <- sharpenGetFrame  src/plugin.cpp:14-76
 *   lgcr_sharpen_destroy  <- sharpenFree      src/plugin.cpp:78-82
 * ------------------------------------------------------------------- */
/* Sharpen arguments, one field per entry of the reference signature
 *   clip:vnode;alpha:float:opt;sigma:float:opt;sratio:float:opt;
 *   gspatial:float:opt;ar:float:opt          (src/plugin.cpp:1172-1176)
 * NaN = not given (defaults 0.3, 0.01, 0.15, 1.2, 0.0). */
typedef struct lgcr_sharpen_params {
    double alpha, sigma, sratio, gspatial, ar;
} lgcr_sharpen_params;

typedef struct lgcr_sharpen lgcr_sharpen;

void lgcr_sharpen_params_init(lgcr_sharpen_params *params);
/* Validates like sharpenCreate and returns LGCR_E_INVALID with its message
 * ("LGCR Sharpen: planar YUV only", "LGCR Sharpen: sigma/sratio/gspatial
 * must be > 0"). fmt->width/height 0 accepts any frame size. */
int lgcr_sharpen_create(const lgcr_sharpen_params *params, const lgcr_format *fmt,
                        lgcr_sharpen **out, char *err, size_t errlen);
void lgcr_sharpen_destroy(lgcr_sharpen *filter);
/* One frame: in/out Y, U, V planes of the clip's format (all three output
 * planes are written). memory as for lgcr_recon_frame: LGCR_MEM_HOST
 * uploads, runs, downloads and returns when done; LGCR_MEM_DEVICE enqueues
 * on `stream` without waiting. Safe to call from several host threads. */
int lgcr_sharpen_frame(lgcr_sharpen *filter, const lgcr_plane in[3], const lgcr_plane out[3],
                       int memory, void *stream);

/* ---------------------------------------------------------------------
 * TRecon: motion-compensated temporal Recon (same-size 4:2:0/4:2:2/4:4:4
 * -> 4:4:4, lanczos3 base, algo 2). Each frame is reconstructed with the
 * chroma samples of its temporal neighbours as extra taps, after 16x16
 * block matching on luma and a chroma-consistency check per block.
 *   lgcr_trecon_create    <- tReconCreate     src/plugin.cpp:920-990
 *   lgcr_trecon_neighbors <- temporalFrameNumbers src/plugin.cpp:729-738
 *   lgcr_trecon_frame     <- tReconGetFrame   src/plugin.cpp:740-918
 *   lgcr_trecon_destroy   <- lgcrFree         src/plugin.cpp:992-996
 * ------------------------------------------------------------------- */
/* TRecon arguments, one field per entry of the reference signature
 *   clip:vnode;strength:float:opt;sigma:float:opt;sratio:float:opt;
 *   sdb:float:opt;gsigma:float:opt;stretch:float:opt;ar:float:opt;
 *   ridge:int:opt;sparse:int:opt;ms:float:opt;trad:int:opt;
 *   tsearch:int:opt;tsad:float:opt;bm:int:opt  (src/plugin.cpp:1177-1181)
 * Doubles NaN and ints LGCR_UNSET_INT mean "not given". */
typedef struct lgcr_trecon_params {
    double strength, sigma, sratio, sdb, gsigma, stretch, ar;
    int ridge, sparse;
    double ms;
    int trad, tsearch;
    double tsad;
    int bm;
} lgcr_trecon_params;

typedef struct lgcr_trecon lgcr_trecon;

void lgcr_trecon_params_init(lgcr_trecon_params *params);
/* Validates like tReconCreate (the clip's frame count is num_frames) and
 * returns LGCR_E_INVALID with its message on failure. */
int lgcr_trecon_create(const lgcr_trecon_params *params, const lgcr_format *fmt,
                       int num_frames, lgcr_trecon **out, char *err, size_t errlen);
void lgcr_trecon_destroy(lgcr_trecon *filter);
/* Frame numbers frame n needs besides itself, in the order
 * lgcr_trecon_frame expects them (n +- trad clamped to the clip, without n,
 * without repeats). Returns their count (at most 2 * trad); frames holds up
 * to cap of them. */
int lgcr_trecon_neighbors(const lgcr_trecon *filter, int n, int *frames, int cap);
/*
 * One frame: cur[0..2] the frame's Y, U, V; nbrs[3*k .. 3*k+2] the planes of
 * the k-th neighbour from lgcr_trecon_neighbors (count of them; ignored when
 * strength is 0); out[0..2] 4:4:4 Y, U, V (all written). chroma_location,
 * memory and stream as for lgcr_recon_frame.
 */
int lgcr_trecon_frame(lgcr_trecon *filter, const lgcr_plane cur[3], const lgcr_plane *nbrs,
                      int count, const lgcr_plane out[3], int chroma_location, int memory,
                      void *stream);

/* ---------------------------------------------------------------------
 * Downsample: the reference's fourth filter, 4:4:4 -> 4:2:0 (8-16 bit or
 * float). A separable polyphase base (spline36, lanczos3 or binomial) with
 * a luma-guided correction near structure: quality 0 and 1 average the
 * chroma along the luma's edge direction, quality 2 also scores four
 * candidates by how well they re-upsample to the source chroma.
 *   lgcr_downsample_create  <- downsampleCreate   src/downsample.cpp:820-911
 *   lgcr_downsample_frame   <- downsampleGetFrame src/downsample.cpp:740-781
 *   lgcr_downsample_destroy <- downsampleFree     src/downsample.cpp:814-818
 * ------------------------------------------------------------------- */
/* Downsample arguments, one field per entry of the reference signature
 *   clip:vnode;quality:int:opt;kernel:data:opt;strength:float:opt;
 *   loc:data:opt                       (src/downsample.cpp:913-918)
 * quality LGCR_UNSET_INT, kernel / loc NULL and strength_set 0 mean "not
 * given" (defaults 0, "spline36", 1.0, "left"); a given strength, NaN
 * included, is validated like the reference's. */
typedef struct lgcr_downsample_params {
    int quality;
    const char *kernel;       /* "spline36", "lanczos3" or "binomial"     */
    double strength;
    int strength_set;
    const char *loc;          /* "left", "center", "topleft", "top",
                                 "bottomleft" or "bottom"                  */
} lgcr_downsample_params;

typedef struct lgcr_downsample lgcr_downsample;

void lgcr_downsample_params_init(lgcr_downsample_params *params);
/* Validates like downsampleCreate (planar YUV 4:4:4, 8-16 bit integer or
 * 32-bit float, even width and height: fmt->width/height must be given) and
 * returns LGCR_E_INVALID with its message ("Downsample: input must be planar
 * YUV444 (8-16 bit integer or float32)", ...). */
int lgcr_downsample_create(const lgcr_downsample_params *params, const lgcr_format *fmt,
                           lgcr_downsample **out, char *err, size_t errlen);
void lgcr_downsample_destroy(lgcr_downsample *filter);
/* The _ChromaLocation the output frames carry (0 left .. 5 bottom). */
int lgcr_downsample_chroma_location(const lgcr_downsample *filter);
/*
 * One frame: in[0..2] the 4:4:4 Y, U, V planes; out[1], out[2] the
 * (width/2) x (height/2) U and V planes. out[0].data NULL leaves luma to the
 * caller (the reference shares the source's Y plane with the output frame);
 * otherwise Y is copied to out[0]. memory and stream as for lgcr_recon_frame.
 */
int lgcr_downsample_frame(lgcr_downsample *filter, const lgcr_plane in[3], const lgcr_plane out[3],
                          int memory, void *stream);

/* ---------------------------------------------------------------------
 * Batched form: many frames (any mix of filters, sizes, subsamplings and
 * depths) in one launch per pipeline stage, captured as a CUDA graph and
 * replayed when the same batch layout is submitted again.
 * ------------------------------------------------------------------- */
typedef struct lgcr_batch lgcr_batch;

typedef struct lgcr_batch_item {
    lgcr_recon *filter;
    lgcr_plane in[3];        /* device memory */
    lgcr_plane out[3];       /* device memory */
    int chroma_location;
} lgcr_batch_item;

int lgcr_batch_create(lgcr_batch **out);
void lgcr_batch_destroy(lgcr_batch *batch);
/* Enqueue all items on `stream`; returns without waiting. use_graph != 0
 * captures the launch sequence into a CUDA graph on first use of a layout
 * and replays it afterwards. */
int lgcr_batch_run(lgcr_batch *batch, const lgcr_batch_item *items, int count,
                   void *stream, int use_graph);
/* Number of kernel launches the last lgcr_batch_run enqueued. */
int lgcr_batch_launch_count(const lgcr_batch *batch);

/* Stage profiling (the reference's per-stage PipelineMetrics timers,
 * src/pipeline.h:315-388, as CUDA events): when on, every stage launch of
 * later runs is bracketed by events (graph replay is bypassed). */
int lgcr_batch_set_profiling(lgcr_batch *batch, int on);
/* Accumulated device ms and launch counts per stage since the last reset;
 * waits for the recorded work. Arrays have lgcr_stage_count() entries. */
int lgcr_batch_stage_times(lgcr_batch *batch, double *ms, int *launches, int reset);
int lgcr_stage_count(void);
const char *lgcr_stage_name(int stage);

/* Per-batch autotuner: on the given items (the layout about to be run),
 * times the candidate block shapes of the tunable per-pixel stages, the
 * guided kernel's variants and the frame grouping of the stage sequence,
 * and keeps the fastest for this batch only (later runs of `batch` use
 * them; other batches and the per-frame path are unaffected). Runs the
 * items several times on `stream` and waits for them; report (optional)
 * receives one line per tuned choice. */
int lgcr_batch_autotune(lgcr_batch *batch, const lgcr_batch_item *items, int count,
                        void *stream, char *report, size_t reportlen);

/* Autotuner: time the candidate launch shapes of every stage on the
 * given items and keep the fastest per stage (process-wide: frames planned
 * afterwards use them; plans already made keep the settings they were
 * planned with). */
int lgcr_autotune(const lgcr_batch_item *items, int count, void *stream,
                  char *report, size_t reportlen);

/* ---------------------------------------------------------------------
 * Serving form: a request loop with continuous batching under a device
 * memory budget. Requests carry host planes; each stream key keeps its
 * device-resident tables and workspaces.
 * ------------------------------------------------------------------- */
typedef struct lgcr_server lgcr_server;

typedef struct lgcr_server_config {
    size_t device_budget_bytes;   /* admission budget for workspaces      */
    int max_batch;                /* frames per device batch (>=1)        */
    int lanes;                    /* concurrent device streams (>=1)      */
    int queue_capacity;           /* pending requests before LGCR_E_BUSY  */
} lgcr_server_config;

typedef struct lgcr_request_info {
    int status;
    double submit_ms, start_ms, done_ms;   /* server clock, milliseconds */
    int batch_size;                        /* frames in its device batch  */
} lgcr_request_info;

int lgcr_server_create(const lgcr_server_config *config, lgcr_server **out);
/* Submit one frame. Host planes must stay valid until completion.
 * Returns a ticket (>=0) or a negative status. */
int64_t lgcr_server_submit(lgcr_server *server, lgcr_recon *filter,
                           const lgcr_plane in[3], const lgcr_plane out[3],
                           int chroma_location);
/* Wait for a ticket (timeout_ms < 0 waits without limit). */
int lgcr_server_wait(lgcr_server *server, int64_t ticket, int timeout_ms,
                     lgcr_request_info *info);
/* Hold (on != 0) or release admission of queued requests (host-side
 * control used to exercise bounded waits and admission). */
int lgcr_server_pause(lgcr_server *server, int on);
void lgcr_server_destroy(lgcr_server *server);

#ifdef __cplusplus
}
#endif

#endif /* LGCR_B200_H */
