/* fdv_b200 -- the fdv encoder analysis loop on NVIDIA B200 (sm_100a).
 *
 * A drop-in for the encode side of the fdv codec (yhbsh/fdv, include/fdv.h):
 * the same entry points, argument meanings, return conventions and byte
 * streams, with the per-frame analysis loop -- motion search, motion
 * compensation, the 4x4/8x8 transforms with quantisation and RDOQ, mode
 * decision, reconstruction and deblocking -- running as CUDA kernels, and the
 * rANS / adaptive entropy coding of the decided symbols on the host.
 *
 * Every function here is a plain C symbol of libfdvb200.so.  Pointers are host
 * pointers; frames are I420 (w*h luma bytes, then (w/2)*(h/2) U, then V).
 * Functions that return a size return 0 on error; functions that return int
 * return 0 on success and a negative value on error; fdvb_last_error() then
 * describes the failure.  Nothing aborts the process.
 *
 * Streams are byte-identical to the reference encoder's for the same frames,
 * QP, key interval, band layout and motion search range.  The reference fixes
 * its search range at compile time (FDV_ME_RANGE, fdv.h:5163-5170; 16 by
 * default); fdvb_set_search_range() is the run-time equivalent. */
#ifndef FDV_B200_H
#define FDV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------ the fdv.h encode API -- */

/* Encode nframes I420 frames as one video stream.  Replaces
 * fdv_video_encode, fdv.h:903 (implementation fdv.h:6741-6854).  frame f is a
 * key frame iff f == 0 or (keyint > 0 && f % keyint == 0); keyint is clamped
 * to 0..255.  w and h must be multiples of 16.  Returns the stream length, or
 * 0 on error (bad arguments, out of room, device failure). */
size_t fdv_video_encode(const uint8_t *const *frames, int nframes, int w, int h, int qp, int keyint,
                        uint8_t *out, size_t cap);

/* Encode as a tile-parallel container of independent horizontal bands of
 * band_mbrows macroblock rows.  Replaces fdv_vtile_encode, fdv.h:973
 * (implementation fdv.h:7161-7243).  All bands are analysed together on the
 * GPU; nthreads bounds the host threads used for entropy coding and never
 * changes the output. */
size_t fdv_vtile_encode(const uint8_t *const *frames, int nframes, int w, int h, int qp, int keyint,
                        int band_mbrows, int nthreads, uint8_t *out, size_t cap);

/* The GPU decoder.  Replaces fdv_video_decode, fdv.h:907 (implementation
 * fdv.h:6856-6930) and fdv_vtile_decode, fdv.h:980 (implementation
 * fdv.h:7245-7370), same signatures: nframes consecutive I420 frames into out,
 * which must hold them.  The frame blobs are entropy-decoded and parsed on the
 * host -- entropy decoding by one chain per band, records by a worker pool,
 * nthreads threads in all at most -- running up to three frames ahead of the
 * GPU; prediction, inverse transforms, deblocking
 * and reference preparation run on the GPU, bit-exact with the reference
 * decoder.
 * Returns 0, or -1 for a malformed stream or a device failure (the reason:
 * fdvd_last_error).  Motion vectors are bounds-checked against the border the
 * reference decoder built for the current search range (16 -> 32 samples,
 * 32 -> 64, 64 -> 96), so a stream decodes here exactly when it decodes
 * there.  The output never depends on nthreads. */
int fdv_video_decode(const uint8_t *in, size_t len, uint8_t *out, int *nframes, int *w, int *h);
int fdv_vtile_decode(const uint8_t *in, size_t len, uint8_t *out, int *nframes, int *w, int *h, int nthreads);
/* The reason the last fdv_*_decode call on this thread failed ("" if none). */
const char *fdvd_last_error(void);
/* Decoder timing, off by default (no counterpart in the reference): with it on,
 * CUDA events on the decoder's compute stream bracket each launch and the host
 * stages are clocked.  fdvd_stats reads the milliseconds ms[k] and counts n[k]
 * accumulated since the last reset, k = 0 P-frame inter reconstruction,
 * 1 INTRA16 reconstruction, 2 key-frame reconstruction, 3 deblocking +
 * reference preparation, 4 whole frame steps on the compute stream (launches);
 * host wall time of 5 entropy decoding (summed over the per-band chains),
 * 6 scattering decoded frames into the output (summed over the copier
 * threads), 7 the submitting thread waiting for parsed frames, 8 building
 * records from symbols (summed over the record workers) (counts: frames);
 * reset != 0 clears them. */
void fdvd_timing(int on);
void fdvd_stats(double ms[9], long long n[9], int reset);
/* Host timing of the last whole-array encode (fdv_video_encode or
 * fdv_vtile_encode; no counterpart in the reference), milliseconds since the
 * call entered the encoder: ms[0] the first submission to the GPU, ms[1] the
 * last frame collected, ms[2] the end of the last entropy coding, ms[3] the
 * end; ms[4] the calling thread's summed waits in collects, ms[5] its summed
 * time in the band-parallel entropy coding. */
void fdvb_encode_stats(double ms[6]);

/* Streaming encoder.  Replaces the fdv_enc_* family, fdv.h:1157-1198
 * (implementation fdv.h:8129-8459).  Output is byte-identical to
 * fdv_video_encode (or fdv_vtile_encode for a tiled encoder) over the same
 * frames. */
typedef struct fdv_encoder fdv_encoder;
fdv_encoder *fdv_enc_open(int w, int h, int qp, int keyint);                       /* fdv.h:1160 */
fdv_encoder *fdv_enc_open_tiled(int w, int h, int qp, int keyint, int band_mbrows,
                                int nthreads);                                     /* fdv.h:1186 */
int fdv_enc_frame(fdv_encoder *e, const uint8_t *i420);                           /* fdv.h:1163 */
int fdv_enc_repeat(fdv_encoder *e);                                                /* fdv.h:1169 */
/* Switch an encoder to average-bitrate control before its first frame.
 * Replaces fdv_enc_set_bitrate, fdv.h:1176 (implementation :8385-8392).  A
 * single-stream encoder codes each P-frame at a real operating point (QP plus
 * a lambda fraction) and codes a frame again, coarser, up to three times when
 * it lands more than 1.5x over its allocation (fdv.h:8281-8335); a tiled
 * encoder hands every band the same whole QP per frame (fdv.h:8076-8083).
 * Returns -1 after the first frame or for a non-positive bitrate. */
int fdv_enc_set_bitrate(fdv_encoder *e, int bits_per_second, int fps, double bufsecs);
int fdv_enc_count(const fdv_encoder *e);                                           /* fdv.h:1189 */
size_t fdv_enc_bytes(const fdv_encoder *e);                                        /* fdv.h:1190 */
uint8_t *fdv_enc_finish(fdv_encoder *e, int fps, size_t *len);                    /* fdv.h:1195 */
void fdv_enc_close(fdv_encoder *e);                                                /* fdv.h:1198 */

/* The rate controller itself (fdv.h:1022-1053), for callers that drive
 * fdv_video_encode-style loops themselves.  Same fields and semantics as the
 * reference's fdv_rc. */
typedef struct {
    int bitrate;             /* bits per second, the average to hold */
    int fps;
    double bufbits;          /* bucket size */
    int qpmin, qpmax, keyint;
    double qp_p;             /* the P-frame operating point */
    double ip_off;           /* how much finer a key frame is coded */
    double last_target;      /* the last frame's allocation, bits */
    double fill;             /* bucket fullness, bits */
    int used_qp;
    double lscale;           /* the operating point's fraction, as a lambda multiplier */
} fdv_rc;
void fdv_rc_init(fdv_rc *rc, int bitrate, int fps, int w, int h, int keyint, double bufsecs, int qpmin,
                 int qpmax);                                                   /* fdv.h:1036 */
int fdv_rc_pick(fdv_rc *rc, int is_intra);                                     /* fdv.h:1038 */
void fdv_rc_update(fdv_rc *rc, int is_intra, size_t bytes);                    /* fdv.h:1039 */
void fdv_rc_skip(fdv_rc *rc, size_t bytes);                                    /* fdv.h:1044 */
void fdv_rc_adopt(fdv_rc *rc, int is_intra, double q);                         /* fdv.h:1051 */
void fdv_rc_split(const fdv_rc *rc, double q, int *qp, double *lscale);        /* fdv.h:1053 */

/* The 12-byte .fdv file head.  Replaces fdv_wrap, fdv.h:1094. */
size_t fdv_wrap(uint8_t *out, size_t cap, int kind, int fps, const uint8_t *payload, size_t payload_len);

/* ---------------------------------------------------------- settings -- */

/* Motion search radius in pels: 16 (the reference's default), 32 or 64.
 * The run-time form of FDV_ME_RANGE (fdv.h:5169).  Returns the previous
 * value, or -1 for an unsupported radius.  Affects encoders opened after the
 * call. */
int fdvb_set_search_range(int range);
int fdvb_get_search_range(void);
/* CUDA device used by encoders opened after the call (default 0). */
int fdvb_set_device(int device);
/* Description of the last failure on the calling thread. */
const char *fdvb_last_error(void);
/* fdv_video_encode and fdv_vtile_encode, and the two decoders, each keep up to
 * four GPU engines (device and pinned memory for one frame geometry) between
 * calls so that repeated calls skip the set-up; this frees them.  No
 * counterpart in the reference. */
void fdvb_release_engines(void);

/* -------------------------------------------- the inner engine ABI -- */

/* A batch of independent encoder units (bands of a stream, or streams),
 * advanced one frame per call.  This is the seam that replaces the body of
 * the reference's static pframe_encode macroblock loop and deblock
 * (fdv.h:5797-6170) and fdv_image_encode's intra walk and deblock
 * (fdv.h:4849-4879): the analysis runs on the GPU and each unit's decided
 * symbols come back as the byte streams the reference's entropy tail
 * (fdv.h:6172-6426 and :4881-5032) partitions and codes. */
typedef struct fdvb_engine fdvg_ctx;
fdvg_ctx *fdvg_create(int nunits, const int *w, const int *h, int range, int device);
void fdvg_destroy(fdvg_ctx *g);
/* One frame for every unit.  planes[3*u + p] is unit u's plane p (Y, U, V),
 * rows contiguous (stride w, w/2, w/2); all may be NULL for a held frame
 * (force_skip[u] != 0, fdv_enc_repeat).  is_intra[u] selects a key frame.
 * lscale may be NULL (1.0: the fractional-lambda multiplier of fdv.h:5804). */
int fdvg_frame(fdvg_ctx *g, const uint8_t *const *planes, const int *is_intra, const int *qp,
               const double *lscale, const int *force_skip);
/* fdvg_frame in two halves, so a host can entropy-code one frame while the GPU
 * analyses the next: fdvg_submit copies the sources (through pinned staging;
 * the caller may reuse its buffers on return) and queues the frame; at most
 * 60 frames are in flight.  fdvg_collect waits for the oldest one, after
 * which the stream and count accessors describe it until the next
 * fdvg_collect.  A collected frame's streams stay valid until the next
 * submission. */
int fdvg_submit(fdvg_ctx *g, const uint8_t *const *planes, const int *is_intra, const int *qp,
                const double *lscale, const int *force_skip);
int fdvg_collect(fdvg_ctx *g);
/* Up to fdvg_max_batch(g) consecutive P-frames in one submission (sixty by
 * default, fdvg_set_tuning; one while decision records or deferred references
 * are on):
 * the arrays hold frame k's entries at k * nunits (planes: 3 per unit).  The
 * frames' wavefronts run in one launch, each frame's macroblock rows starting
 * as soon as the reference tiles they read have been written by the frame
 * before (deblocked and prepared inside the wavefront); the frames are then
 * collected one by one as after fdvg_submit, with the same streams as
 * frame-by-frame coding. */
int fdvg_submit_batch(fdvg_ctx *g, int nframes, const uint8_t *const *planes, const int *is_intra, const int *qp,
                      const double *lscale, const int *force_skip);
int fdvg_max_batch(const fdvg_ctx *g);
/* The engine's launch shape, the autotuner's knobs (no counterpart in the
 * reference): max_batch P-frames per launch at most (1..60) and p_grid blocks
 * of the P-frame wavefront kernel, i.e. macroblock rows in flight (0: one per
 * SM; capped at the SM count).  fdvg_get_tuning reports the shape in force and
 * the SM count.  fdvb_set_tuning records a shape for every engine the fdv_*
 * encoders create or reuse for that geometry (units of w[i] x h[i] at search
 * range `range`); max_batch 0 removes the record.  Returns 0 or -1. */
int fdvg_set_tuning(fdvg_ctx *g, int max_batch, int p_grid);
/* Key-frame lookahead (no counterpart in the reference: the reference codes
 * its frames in order).  A key frame's analysis reads nothing but its own
 * source, and one key frame's CTU-row chains keep few SMs busy, so the next
 * key frame of a sequence can be analysed in the same launch.  Arms `planes`
 * (3 per unit, host or device pointers as the engine's sources) and `qp` (one
 * per unit) for the next key-frame submission of every unit: that launch also
 * analyses and deblocks this frame into a lookahead lane, and when this frame
 * is later submitted as a key frame with the same plane pointers and
 * quantisers, only its symbols are compacted and its reference prepared.  The
 * planes must stay valid and unchanged until that submission; any other key
 * frame drops the analysed one.  NULL planes disarm.  The streams are the
 * same as without it.  fdvg_frames_device, fdv_video_encode and
 * fdv_vtile_encode arm it themselves. */
int fdvg_key_lookahead(fdvg_ctx *g, const uint8_t *const *planes, const int *qp);
void fdvg_get_tuning(const fdvg_ctx *g, int *max_batch, int *p_grid, int *nsm);
int fdvb_set_tuning(int nunits, const int *w, const int *h, int range, int max_batch, int p_grid);
/* nframes frame steps from device sources (planes: 3 * nunits device pointers
 * per frame; is_intra and qp: nunits per frame): runs of P-frames go as
 * batches, each collected while the next one runs.  The stream accessors then
 * describe the last frame. */
int fdvg_frames_device(fdvg_ctx *g, int nframes, const uint8_t *const *dplanes, const int *is_intra, const int *qp);
/* The last frame's symbol streams of unit u.  P-frame: 16 streams in the
 * blob's order (9 structure streams by model, then 4x4 counts, 4x4 levels,
 * 8x8 counts, 8x8 levels, region flags, chroma counts, chroma levels).  Key
 * frame: plane p's 12 streams (split flags of 4 levels, big-leaf modes, the
 * two 4x4 mode contexts, counts, levels, 8x8 counts, 8x8 levels, flags).
 * Pointers stay valid until the next fdvg_frame. */
int fdvg_pframe_streams(fdvg_ctx *g, int u, const uint8_t **s16, size_t *n16);
int fdvg_iframe_streams(fdvg_ctx *g, int u, int plane, const uint8_t **s12, size_t *n12);
/* The per-stream symbol counts of those streams, counted on the GPU while
 * they are compacted: hist[k * 256 + v] is how often byte v occurs in stream
 * k (16 streams for a P-frame, 12 per key-frame plane).  They are the counts
 * the entropy tail builds its rANS tables from (fdv.h:6228-6236,
 * :4899-4905); the library's own tail uses them instead of counting. */
int fdvg_pframe_hist(fdvg_ctx *g, int u, uint32_t *hist);
int fdvg_iframe_hist(fdvg_ctx *g, int u, int plane, uint32_t *hist);
/* The last frame's deblocked reconstruction of unit u (tight I420). */
int fdvg_recon(fdvg_ctx *g, int u, uint8_t *i420);
/* Seed unit u's reference pool (nearest, and optionally the second). */
int fdvg_set_refs(fdvg_ctx *g, int u, const uint8_t *near_i420, const uint8_t *far_i420);
/* fdvg_frame with the planes already in device memory (device pointers, read
 * where they are; they stay unchanged until the call returns). */
int fdvg_frame_device(fdvg_ctx *g, const uint8_t *const *dplanes, const int *is_intra, const int *qp,
                      const double *lscale, const int *force_skip);
/* Device time accumulated since creation or the last reset, measured with
 * CUDA events on the engine's stream: whole steps, the P-frame analysis kernel
 * and the key-frame analysis kernel (with their launch counts), the total
 * number of kernel launches, and the symbol bytes the device wrote to host
 * memory. */
void fdvg_stats(const fdvg_ctx *g, double *step_ms, double *analysis_p_ms, long long *p_launches,
                double *analysis_i_ms, long long *i_launches, long long *kernel_launches, long long *steps,
                long long *d2h_bytes);
void fdvg_stats_reset(fdvg_ctx *g);
/* Bound on one wavefront wait inside the analysis kernels (default 4 s);
 * past it the kernel stops, and fdvg_frame returns an error. */
void fdvg_set_wait_timeout_ns(fdvg_ctx *g, unsigned long long ns);
/* Fault injection for testing the bounded waits: in the next fdvg_frame,
 * P-frame macroblock row `row` of unit u is skipped, so the rows below wait on
 * a progress flag nothing sets; the waits expire and fdvg_frame returns an
 * error, leaving the engine usable. */
void fdvg_inject_stall(fdvg_ctx *g, int u, int row);
/* Per-phase cycle profile of the analysis kernels, for tuning: enable != 0
 * turns it on (thread 0 of every block adds clock64 deltas).  out32 (may be
 * NULL) receives and clears 32 accumulators: [0..9] P-frame kernel (wait,
 * load, SKIP, searches, residuals, region decisions, commit, output,
 * macroblock count, SKIP early-out count); [16..24] key-frame kernel (wait,
 * 4x4 leaves, 8x8/16x16/32x32/64x64 leaves, CTU total, CTU count, 4x4 leaf
 * count). */
int fdvg_phase_profile(fdvg_ctx *g, int enable, unsigned long long *out32);
/* With the phase profile on: the last P-frame's timeline of unit u, two
 * %globaltimer stamps (ns) per macroblock in raster order -- the end of its
 * wait for the row above and its progress publication. */
int fdvg_mb_timeline(fdvg_ctx *g, int u, unsigned long long *out);

/* Allocation-free P-frame analysis of one unit.  No counterpart in the
 * reference.  For callers that cannot allocate device memory while they
 * encode -- a host that owns the GPU's memory pool itself, a real-time path
 * that cannot take cudaMalloc's implicit synchronisation mid-frame -- this
 * runs the same analysis as fdvg_frame (reference preparation, the macroblock
 * wavefront, deblocking, symbol compaction) for one w x h unit with all its
 * scratch in a fixed device array inside the library: 24 MiB
 * (fdvg_pframe_static_capacity), enough for one 1280x720 unit at any search
 * range, held by every GPU that loads the library until the process exits.
 * Larger units are rejected with an error.  The call allocates nothing.
 *
 * cur, near_ref, far_ref (NULL: one reference) and rec are device pointers to
 * tight I420 frames of the unit; rec receives the deblocked reconstruction.
 * out (device memory, out_cap bytes) receives uint32 len[16] followed by the
 * 16 P-frame symbol streams back to back, in fdvg_pframe_streams' order; the
 * streams are assembled in place, so out must be device memory, not
 * host-mapped.  Every pointer must be 16-byte aligned (a misaligned one is
 * rejected before anything is queued).  An out_cap too small for the streams
 * is reported as "output buffer too small ...".  stream is a cudaStream_t
 * (NULL: the default stream); the call synchronises it before returning 0, or
 * a negative value with fdvg_pframe_static_error() set.
 *
 * The first call on a device looks up the array's device address and uploads
 * the transform tables with that device current; make it before any stream
 * capture.  Every call shares the one array and leaves its contents behind:
 * calls that overlap on the GPU (other threads, other streams of the same
 * device) race on it and must be serialised by the caller. */
int fdvg_pframe_static(const uint8_t *cur, const uint8_t *near_ref, const uint8_t *far_ref, uint8_t *rec, int w,
                       int h, int qp, double lscale, int range, uint8_t *out, size_t out_cap, void *stream);
size_t fdvg_pframe_static_capacity(void);
const char *fdvg_pframe_static_error(void);

/* --------------------------------------------- the host entropy tail -- */

/* Entropy state carried between P-frames (fdv.h:590-601). */
typedef struct fdvb_tabcache fdvb_tabcache;
fdvb_tabcache *fdvb_tabcache_new(void);
void fdvb_tabcache_reset(fdvb_tabcache *tc);
void fdvb_tabcache_free(fdvb_tabcache *tc);
/* A P-frame blob from its 16 streams (fdv.h:6172-6426). */
size_t fdvb_entropy_pframe(const uint8_t *const *s16, const size_t *n16, int qp, fdvb_tabcache *tc,
                           uint8_t *out, size_t cap);
/* An intra plane blob from its 12 streams (fdv.h:4881-5032). */
size_t fdvb_entropy_image(const uint8_t *const *s12, const size_t *n12, int w, int h, int qp,
                          uint8_t *out, size_t cap);

/* ------------------------------------------------------ measurement -- */

/* 32-bit integer lane-operations per second the device retires (best of reps
 * timed launches of independent multiply-add / add chains over every SM):
 * the measured denominator of the analysis kernels' integer-op roofline.  No
 * counterpart in the reference.  Returns 0 on error. */
double fdvb_measure_int_rate(int device, int reps);

/* -------------------------------------------- synthetic test content -- */

/* Seeded moving-rectangle content: band-limited noise background (sigma 3 px,
 * luma mean 128 / sd 30, chroma sd 10), nrects textured rectangles with sides
 * in [rect_min, rect_max] moving at up to vmax_qpel quarter-pels per frame per
 * axis, a global pan of (pan_qx, pan_qy) quarter-pels per frame, and a fixed
 * textured region over static_pct % of the frame. */
typedef struct fdvb_scene_state fdvb_scene_state;
typedef struct fdvb_scene_params {
    int w, h, nframes;
    int nrects, rect_min, rect_max;
    int vmax_qpel;
    int pan_qx, pan_qy;
    int static_pct;
    unsigned long long seed;
} fdvb_scene_params;
fdvb_scene_state *fdvb_scene_open(const fdvb_scene_params *params);
int fdvb_scene_frame(const fdvb_scene_state *s, int f, uint8_t *i420);
void fdvb_scene_close(fdvb_scene_state *s);

/* Camera-like stress content: a fractal canvas (value-noise octaves with
 * amplitude proportional to wavelength: a 1/f^2 power spectrum; luma mean 128
 * / sd 40, chroma sd 14) seen through a window that pans by (pan_qx, pan_qy)
 * quarter-pels per frame and zooms by zoom_ppm parts per million per frame
 * (in on even segments, out on odd ones); nobjects textured objects with sides
 * in [obj_min, obj_max] moving at up to vmax_qpel quarter-pels per frame per
 * axis; additive noise of sd noise_y_x16 / 16 on luma and noise_c_x16 / 16 on
 * chroma; a hard cut to a new canvas and new objects every cut_every frames
 * (0: never).  Integer arithmetic: the same bytes on every machine.  Frames
 * may be rendered from several threads at once. */
typedef struct fdvb_camscene_state fdvb_camscene_state;
typedef struct fdvb_camscene_params {
    int w, h, nframes;
    int nobjects, obj_min, obj_max;
    int vmax_qpel;
    int zoom_ppm;
    int pan_qx, pan_qy;
    int noise_y_x16, noise_c_x16;
    int cut_every;
    unsigned long long seed;
} fdvb_camscene_params;
fdvb_camscene_state *fdvb_camscene_open(const fdvb_camscene_params *params);
int fdvb_camscene_frame(const fdvb_camscene_state *s, int f, uint8_t *i420);
void fdvb_camscene_close(fdvb_camscene_state *s);


/* ---- Learned proposal network (no counterpart in the reference) ----------
 * A 4-layer convolutional network (140,203 parameters; bf16 on the tensor
 * cores, fp32 master weights and accumulation) that proposes four motion
 * vectors and a SKIP / inter / intra prior per macroblock.  It is trained on
 * (macroblock, chosen MV, chosen mode, RD cost) tuples of the plain encoder.
 * Training samples index a bank of luma planes on the device.  All functions
 * return 0 or -1 (fdvl_last_error() says why). */
typedef struct fdvl_net fdvl_net;
typedef struct {
    int cur, ref;        /* bank slots of the current and the nearest reference luma */
    int mbx, mby;        /* macroblock */
    int cls;             /* 0 SKIP, 1 inter (INTER16 / INTER8), 2 intra */
    int has_mv;          /* mvx/mvy is a target (inter on the nearest reference) */
    int mvx, mvy;        /* quarter-pel */
    int qp;              /* the frame's quantiser (an input of the network) */
    float weight;
} fdvl_sample;
int fdvl_nparams(void);
fdvl_net *fdvl_create(int device, int max_batch, int bank_frames, int w, int h);
void fdvl_destroy(fdvl_net *n);
int fdvl_set_params(fdvl_net *n, const float *p);   /* also resets the Adam state */
int fdvl_get_params(fdvl_net *n, float *p);
int fdvl_bank_put(fdvl_net *n, int slot, const uint8_t *y);
/* Input features (n x 32 x 32 x 4) and outputs (n x 16: 8 MV coordinates in
 * units of 16 quarter-pels, 3 mode logits, 5 zero) of n samples. */
int fdvl_features(fdvl_net *n, const fdvl_sample *s, int nb, float *x);
int fdvl_forward(fdvl_net *n, const fdvl_sample *s, int nb, float *out);
/* The same through the fused per-frame inference kernel the encoder uses,
 * plus its per-macroblock proposals (20 bytes each: four quarter-pel vectors
 * as int16 x/y pairs clamped to +-lim, then the confident class as int32,
 * -1 when the mode softmax stays below conf). */
int fdvl_forward_fused(fdvl_net *n, const fdvl_sample *s, int nb, float conf, int lim, float *out, void *hints);
/* Per-phase cycle sums of the fused inference kernel, for tuning (enable
 * turns the counters on; out16 receives and clears them): staging, features,
 * conv1, its epilogue, conv2, its epilogue, conv3, fc, then the group count. */
int fdvl_infer_profile(fdvl_net *n, int enable, unsigned long long *out16);
/* Gradient of the batch-mean loss (nb a multiple of 64); loss[3] = total, mode, MV. */
int fdvl_grads(fdvl_net *n, const fdvl_sample *s, int nb, float *grad, float *loss);
int fdvl_train_step(fdvl_net *n, const fdvl_sample *s, int nb, float lr, float *loss);
/* Adam over shuffled batches with a cosine-decayed rate; curve[2*epochs]
 * (mode, MV loss per epoch, sampled) may be NULL. */
int fdvl_train(fdvl_net *n, const fdvl_sample *s, int ns, int batch, int epochs, float lr, unsigned long long seed,
               float *curve);
const char *fdvl_last_error(void);
/* One D[M][N] = A[M][K] * B[N][K]^T through the network's tcgen05 GEMM
 * (A, B bf16 bit patterns, row-major; K a multiple of 64*nsplit). */
int fdvl_gemm(int device, int M, int N, int K, const uint16_t *A, const uint16_t *B, float *D, int nsplit);

/* The learned-proposal form of the encoder.  With proposals on, every P-frame
 * first runs the network over all its macroblocks (one inference per frame
 * step); where the mode prior's softmax reaches `conf`, the macroblock's
 * analysis is narrowed: SKIP / inter search the nearest reference's 16x16
 * vector from the four proposed vectors (a few diamond steps, then the
 * sub-pel refinement) and skip the second reference, the INTER8 chain and
 * intra; intra skips the motion searches.  Elsewhere the full search runs.
 * The streams stay valid fdv streams (the decoder does not care how a mode
 * was chosen) but are no longer byte-identical to the reference encoder's.
 * params: fdvl_nparams() floats; NULL turns proposals off.  This call sets
 * the product configuration: the SKIP class at threshold `conf`, taken only
 * while the best merge candidate's RD cost is at most 400 lambda; the inter
 * class at `conf` too, its narrowed analysis keeping INTER8 (four seeded,
 * shortened 8x8 searches); the intra class at `conf`.  Every full search starts
 * its motion searches from the proposed vectors too (doubled for the second
 * reference).  fdvg_set_learned_conf changes it. */
int fdvg_set_learned(fdvg_ctx *g, const float *params, float conf);
/* conf5: per-class thresholds (SKIP, inter, intra) in place of the single
 * one -- a value above 1 keeps that class on the full search --, a SKIP gate
 * (a confident SKIP is taken only while the best merge candidate's RD cost
 * is at most gate * lambda; gate <= 0: no gate) and, when nonzero, INTER8 in
 * the confident-inter path (its four searches seeded with the proposals and
 * cut to a few diamond steps). */
int fdvg_set_learned_conf(fdvg_ctx *g, const float *conf5);
/* The process-wide setting used by fdv_video_encode / fdv_vtile_encode /
 * fdv_enc_* from the next call on. */
int fdvb_set_learned(const float *params, float conf);
/* Per-macroblock decision records of the last collected P-frame (for
 * building training tuples): mode (0 SKIP, 1 INTER16, 2 INTRA16, 3 INTER8),
 * MV (quarter-pel, the vector neighbours predict from), reference, and RD
 * cost of the chosen mode (fdvg_set_records(g, 1) before the frame).  Any
 * output may be NULL. */
int fdvg_set_records(fdvg_ctx *g, int enable);
int fdvg_mb_records(fdvg_ctx *g, int u, uint8_t *mode, int16_t *mv, uint8_t *ref, float *cost);

#ifdef __cplusplus
}
#endif
#endif /* FDV_B200_H */
