// Internal declarations shared by the host-side translation units of
// libfdvb200: the entropy tail, the container writers, the GPU engine driver
// and the synthetic content generator.  Nothing here is part of the public
// C ABI (include/fdv_b200.h).
#pragma once
#include <cstddef>
#include <cstdint>

#include "../../../include/fdv_b200.h"

// ---------------------------------------------------------------- streams --
// P-frame symbol streams, in the order the frame blob carries them
// (fdv.h:6170-6210): nine structure streams keyed by model (four macroblock
// mode contexts, then reference index, MV x bytes, MV y bytes, intra sub-mode,
// merge index), then the seven coefficient streams.
enum {
    PS_MODE0 = 0, PS_MODE3 = 3,
    PS_REF = 4, PS_MVX = 5, PS_MVY = 6, PS_SUB = 7, PS_MERGE = 8,
    PS_NSTRUCT = 9,
    PS_CN = 9, PS_CL = 10, PS_CN8 = 11, PS_CL8 = 12, PS_CFL = 13, PS_CNC = 14, PS_CLC = 15,
    PS_NS = 16
};

// Intra (image codec) streams of one plane (fdv.h:4273-4289) for a 64x64 CTU:
// split flags of the four node levels, big-leaf mode, the two 4x4 mode
// contexts, then 4x4 counts, 4x4 levels, 8x8 counts, 8x8 levels, region flags.
enum {
    IS_SPLIT0 = 0, IS_MODEB = 4, IS_MODE0 = 5, IS_MODE1 = 6, IS_NSTRUCT = 7,
    IS_CNT = 7, IS_LVL = 8, IS_CNT8 = 9, IS_LVL8 = 10, IS_FLAG = 11, IS_N = 12
};

// The per-encoder entropy state carried between P-frames (fdv.h:590-601):
// the last transmitted tables (cached form) and the symbol-count history that
// primes the adaptive coder.  Reset at every key frame.
struct fdvb_tabcache {
    uint16_t f1[256];
    uint16_t fs[16][256];
    int have;
    uint32_t hist[16][256];
    int hn;
};

// One plane's or one P-frame's analysis output, as byte streams.
struct fdvb_streams {
    const uint8_t *s[16];
    size_t n[16];
    const uint32_t *hist = nullptr;   // [16][256] symbol counts of the streams, when the GPU made them
};

// Entropy tail.  Each returns the blob length or 0 when `cap` is too small.
size_t fdvb_pframe_blob(const fdvb_streams *st, int qp, fdvb_tabcache *tc,
                        uint8_t *out, size_t cap, int *emode_out);
size_t fdvb_image_blob(const fdvb_streams *st, int w, int h, int qp,
                       uint8_t *out, size_t cap, int *emode_out);

// Little-endian / LEB helpers shared by the container writers.
size_t fdvb_put16(uint8_t *b, size_t p, unsigned v);
size_t fdvb_put32(uint8_t *b, size_t p, uint32_t v);
size_t fdvb_leb_put(uint8_t *b, size_t p, uint32_t u);
int fdvb_leb_size(uint32_t u);


// λ of the RD decisions, computed with the host libm exactly as the reference
// does (fdv.h:4870, :5804): lscale * 0.425 * 2^((qp - 12) / 3).
double fdvb_lambda(int qp, double lscale);

// The lambda multiplier spanning one quantiser step of the rate controller
// (FDV_RC_LFRAC, fdv.h:7882-7884).
extern "C" double fdvb_rc_lfrac(void);

// The 8x8 DCT basis and quantiser steps (fdv.h:2597-2612), computed on the
// host with the same libm calls and uploaded to the device.
void fdvb_c8_tables(int32_t c8[64], int32_t qstep8[52]);

// The CUDA device the library's engines open on (fdvb_set_device).
int fdvb_device_setting(void);
// Frees the decoders' cached engines (part of fdvb_release_engines).
void fdvd_release_cached(void);
