// The learned motion/mode proposal network: geometry shared by the training
// kernels, the fused inference kernel and the host driver.
//
// Input per macroblock: 32x32 positions x 4 channels (bf16, (v-128)/64):
//   0  current luma, the macroblock and 8 pixels around it (clamped at the edges)
//   1  nearest reference luma at the same place
//   2  current luma over 64x64 around the macroblock, 2x2-averaged
//   3  nearest reference luma over the same 64x64, 2x2-averaged
// and the quantiser, (qp-26)/8, as a 37th reduction column of the first
// convolution (a per-macroblock term of every output: whether a residual is
// worth its bits depends on it).
// Three 3x3 stride-2 convolutions with ReLU (4->32, 32->64, 64->160 channels;
// 32x32 -> 16x16 -> 8x8 -> 4x4) and one fully connected layer (2560 -> 11):
// four motion-vector hypotheses (x, y in units of 16 quarter-pels) and three
// mode logits (SKIP, inter, intra).  140,203 parameters.
//
// Activations are NHWC.  A convolution's reduction index is
// k = (ky*3 + kx)*Cin + ci, so an im2col row gathers nine contiguous channel
// vectors; the fully connected layer reads the 4x4x160 map flattened NHWC.
#pragma once
#include <cstdint>
#include <vector_types.h>

#include "../../../include/fdv_b200.h"

namespace fdvb {
namespace lrn {

constexpr int kPatch = 32, kChan = 4;
constexpr int kQpCol = 36;   // the first convolution's quantiser column
constexpr int kOut = 11, kOutPad = 16;
constexpr int kMvHyp = 4;

struct LayerGeo {
    int sin, cin, cout;   // input side and channels, output channels
    int k, kp;            // reduction length, padded to a multiple of 64
    int gn;               // GEMM N of the forward pass (cout, padded to 16)
    int nr;               // reduction over cout in the input-gradient GEMM, padded to 64
};
// conv1, conv2, conv3, fc
constexpr LayerGeo kGeo[4] = {
    {32, 4, 32, 37, 64, 32, 64},
    {16, 32, 64, 288, 320, 64, 64},
    {8, 64, 160, 576, 576, 160, 192},
    {4, 160, 11, 2560, 2560, 16, 64},
};
constexpr int sout(int l) { return kGeo[l].sin / 2; }
constexpr int pos_per_mb(int l) { return l < 3 ? sout(l) * sout(l) : 1; }

// fp32 master parameters, flat: W1[32][37] b1[32] W2[64][288] b2[64]
// W3[160][576] b3[160] W4[11][2560] b4[11]
constexpr int w_off(int l) {
    int o = 0;
    for (int i = 0; i < l; ++i) o += kGeo[i].cout * kGeo[i].k + kGeo[i].cout;
    return o;
}
constexpr int b_off(int l) { return w_off(l) + kGeo[l].cout * kGeo[l].k; }
constexpr int kNParams = w_off(4);
constexpr int kWOff[4] = {w_off(0), w_off(1), w_off(2), w_off(3)};
constexpr int kBOff[4] = {b_off(0), b_off(1), b_off(2), b_off(3)};
static_assert(kWOff[1] == 1216 && kWOff[2] == 19712 && kWOff[3] == 112032, "offsets");
static_assert(kNParams == 140203, "parameter count");

// One training or inference sample: where its patch comes from, and (training)
// the encoder's decision it is taught.
struct Sample {
    const uint8_t *cur, *ref;   // luma planes; (0,0) is the first visible pixel
    int cs, rs;                 // strides
    int w, h;                   // visible size (reads clamp to it)
    int bx, by;                 // macroblock origin
    int cls, has_mv;            // mode class 0 SKIP / 1 inter / 2 intra; MV target valid
    float tx, ty, wgt;          // MV target (units of 16 quarter-pels), sample weight
    int qp;
};

// Per-macroblock proposal for the P-frame kernel.
struct Hint {
    short2 mv[kMvHyp];   // quarter-pel candidates (ref 0)
    int cls;             // -1: not confident, run the full search; else the mode class
};

}  // namespace lrn

struct UnitDev;
// A network for training (bank_frames > 0: frame bank, gradients, Adam
// state) or for per-frame inference only (bank_frames == 0).
fdvl_net *lrn_create(int device, int max_batch, int bank_frames, int w, int h);
// Proposals for every macroblock of the listed units (pu[i] = {unit index,
// first macroblock}), enqueued on st; lim clamps the vectors (quarter-pels).
int lrn_infer_units(fdvl_net *n, const UnitDev *units, const int2 *pu, int np, int total, float3 conf, int lim,
                    lrn::Hint *hints, unsigned *err, cudaStream_t st);
int lrn_max_batch(const fdvl_net *n);
unsigned *lrn_err_word(fdvl_net *n);

}  // namespace fdvb
