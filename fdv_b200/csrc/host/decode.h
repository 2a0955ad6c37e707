// The decoder's host half: the frame blobs' entropy decoding and symbol parse,
// restated from the reference decoder (fdv.h:5040-5153, :4586-4640, :5421-5465,
// :6429-6737), producing records the GPU reconstruction kernels consume.
// Parsing depends only on symbols and block positions, never on pixels, so the
// whole frame is parsed before any sample is reconstructed.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "fdvb_internal.h"

namespace fdvb {
namespace dec {

// One P-frame macroblock.  Residual coefficients (dequantisation-ready levels
// in natural order, not zigzag) live in a 384-entry block: luma 8x8 region r
// (raster; the INTER8 quadrant q) at [64 r], as four 4x4 blocks of 16 (raster
// within the region) or one 8x8; chroma plane p at [256 + 64 p], four 4x4
// blocks or one 8x8.
struct PMB {
    uint8_t mode;        // 0 SKIP, 1 INTER16, 2 INTRA16, 3 INTER8
    uint8_t ref;         // reference index (SKIP, INTER16)
    uint8_t sub;         // intra sub-mode (INTRA16)
    uint8_t lfl;         // luma region flags, 2 bits each: 0 none, 1 four 4x4, 2 one 8x8
    uint8_t cfl;         // chroma flags, 2 bits per plane (U, V), same meaning
    uint8_t pad[3];
    int16_t mv[4][2];    // SKIP / INTER16: mv[0]; INTER8: the four quadrants
    int32_t coef;        // first coefficient of this macroblock's block, -1: none
    int32_t pad2;
};
static_assert(sizeof(PMB) == 32, "PMB layout");

// One leaf of a key-frame plane's quadtree, in decode order.
struct Leaf {
    uint16_t x, y;       // position in the plane
    uint8_t n, mode;     // size 4..64; 4x4: mode 0..8, larger: DC/V/H/PLANE
    uint16_t nreg;       // 8x8 regions (n >= 8)
    int32_t coef;        // first coefficient (n*n entries, regions of 64 as above; 4x4: 16)
    int32_t fl;          // first region flag in the plane's flag array (n >= 8)
};
static_assert(sizeof(Leaf) == 16, "Leaf layout");

struct PFrame {
    int qp = 0;
    std::vector<PMB> mbs;           // raster order
    std::vector<int16_t> coef;      // 384 per coded macroblock
    std::vector<int32_t> intra;     // INTRA16 macroblocks, raster order
};

struct IPlane {
    int w = 0, h = 0, qp = 0;
    std::vector<Leaf> leaves;
    std::vector<int32_t> ctu_first; // leaf range of each CTU (raster), plus the end
    std::vector<int16_t> coef;
    std::vector<uint8_t> flags;
};

// The entropy-decoded symbol streams of one blob: stream k is
// buf[base[k] .. base[k] + sn[k]).  Decoding them is the part of the parse
// that is sequential over frames (the P-frame table cache); turning symbols
// into records depends on nothing but the symbols.
struct Syms {
    int qp = 0, w = 0, h = 0;   // w, h: a key-frame plane's dimensions
    std::vector<uint8_t> buf;
    size_t sn[16] = {}, base[16] = {};
};
int pframe_symbols(const uint8_t *in, size_t len, int w, int h, fdvb_tabcache *tc, Syms &out);
int pframe_records(const Syms &s, int w, int h, int border, PFrame &out);
int iplane_symbols(const uint8_t *in, size_t len, int w, int h, Syms &out);
int iplane_records(const Syms &s, IPlane &out);

// A P-frame blob of a w x h unit against references with a `border`-sample
// border (the reference's FDV_BORDER: motion vectors reaching past it are
// rejected, fdv.h:6480).  tc carries the entropy tables between frames.
int parse_pframe(const uint8_t *in, size_t len, int w, int h, int border, fdvb_tabcache *tc, PFrame &out);
// One plane's blob of a key frame (fdv_image_decode's stream); the header's
// dimensions must equal w x h.
int parse_iplane(const uint8_t *in, size_t len, int w, int h, IPlane &out);

}  // namespace dec
}  // namespace fdvb
