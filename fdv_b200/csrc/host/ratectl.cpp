// Average-bitrate control: the reference's leaky-bucket feedback loop
// (fdv.h:7822-8029), restated.  It is host arithmetic in IEEE double with the
// same libm calls in the same order (log2, pow, floor, lround), so on the same
// frames it picks the same quantisers and lambda fractions as the reference
// and the coded streams stay byte-identical.
//
// The loop holds a real-valued operating point for P-frames; its integer part
// is the quantiser the format carries and its fraction scales lambda
// (fdv_rc_split).  Key frames follow the P point minus an adapting offset.
// Each frame's target is an even share of a key-frame interval's budget (the
// key frame counted as FDV_RC_IBOOST P-frames), steered back toward a
// half-full bucket over FDV_RC_DRAIN seconds.
#include <cmath>
#include <cstring>

#include "../../../include/fdv_b200.h"

namespace {
constexpr double kDrain = 2.0;     // FDV_RC_DRAIN, seconds to return to half full
constexpr double kStep = 1.0;      // FDV_RC_STEP, largest P move per frame
constexpr double kIpMax = 8.0;     // FDV_RC_IP_MAX
constexpr double kIBoost = 10.0;   // FDV_RC_IBOOST, a key frame's share in P-frames
constexpr double kGain = 1.0;      // FDV_RC_GAIN, QP steps per doubling of the miss
constexpr double kLFrac = 1.15;    // FDV_RC_LFRAC, lambda multiplier of one QP step

// What a frame may cost (rc_target, fdv.h:7920-7945).
double rc_target(const fdv_rc *rc, int is_intra) {
    const double budget = (double)rc->bitrate / rc->fps;
    const double n = (double)rc->keyint;
    const double denom = kIBoost + (n - 1.0);
    double target = budget * n * (is_intra ? kIBoost : 1.0) / denom;
    target -= (rc->fill - rc->bufbits * 0.5) / (rc->fps * kDrain);
    const double lo = budget * (is_intra ? 1.0 : 0.4);
    const double hi = budget * (is_intra ? n * kIBoost / denom * 2.0 : 2.5);
    if (target < lo) target = lo;
    if (target > hi) target = hi;
    return target;
}
}  // namespace

extern "C" {

double fdvb_rc_lfrac(void) { return kLFrac; }

void fdv_rc_init(fdv_rc *rc, int bitrate, int fps, int w, int h, int keyint, double bufsecs, int qpmin, int qpmax) {
    memset(rc, 0, sizeof *rc);
    rc->bitrate = bitrate > 0 ? bitrate : 1000000;
    rc->fps = fps > 0 ? fps : 30;
    rc->bufbits = rc->bitrate * (bufsecs > 0.0 ? bufsecs : 1.0);
    rc->qpmin = qpmin > 0 ? qpmin : 8;
    rc->qpmax = qpmax > 0 ? qpmax : 51;
    rc->fill = rc->bufbits * 0.5;
    rc->keyint = keyint > 1 ? keyint : rc->fps * 10;
    // starting point from bits per pixel per frame (fdv.h:7905-7912)
    const double bpp = (double)rc->bitrate / rc->fps / ((double)w * h);
    double qp = 26.0 - 6.0 * log2(bpp / 0.03);
    if (qp < rc->qpmin) qp = rc->qpmin;
    if (qp > rc->qpmax) qp = rc->qpmax;
    rc->qp_p = qp;
    rc->ip_off = 0.0;
}

void fdv_rc_split(const fdv_rc *rc, double q, int *qp, double *lscale) {
    if (q < rc->qpmin) q = rc->qpmin;
    if (q > rc->qpmax) q = rc->qpmax;
    const int i = (int)floor(q);
    if (i >= rc->qpmax) { *qp = rc->qpmax; *lscale = 1.0; return; }
    *qp = i;
    *lscale = pow(kLFrac, q - (double)i);
}

int fdv_rc_pick(fdv_rc *rc, int is_intra) {
    rc->last_target = rc_target(rc, is_intra);
    const double q = is_intra ? rc->qp_p - rc->ip_off : rc->qp_p;
    int qp;
    if (is_intra) {
        // key frames take the nearest whole quantiser (their lambda is fixed)
        qp = (int)lround(q);
        if (qp < rc->qpmin) qp = rc->qpmin;
        if (qp > rc->qpmax) qp = rc->qpmax;
        rc->lscale = 1.0;
    } else {
        fdv_rc_split(rc, q, &qp, &rc->lscale);
    }
    rc->used_qp = qp;
    return qp;
}

void fdv_rc_adopt(fdv_rc *rc, int is_intra, double q) {
    if (is_intra) {
        double off = rc->qp_p - q;
        if (off < 0.0) off = 0.0;
        if (off > kIpMax) off = kIpMax;
        rc->ip_off = off;
    } else {
        if (q < rc->qpmin) q = rc->qpmin;
        if (q > rc->qpmax) q = rc->qpmax;
        rc->qp_p = q;
    }
}

void fdv_rc_update(fdv_rc *rc, int is_intra, size_t bytes) {
    const double bits = (double)bytes * 8.0;
    const double err = log2(bits / (rc->last_target > 1.0 ? rc->last_target : 1.0));
    double dq = kGain * err;
    if (is_intra) {
        // a key frame moves the offset, not the operating point
        if (dq > 2.0) dq = 2.0;
        if (dq < -2.0) dq = -2.0;
        rc->ip_off -= dq;
        if (rc->ip_off < 0.0) rc->ip_off = 0.0;
        if (rc->ip_off > kIpMax) rc->ip_off = kIpMax;
    } else {
        if (dq > kStep) dq = kStep;
        if (dq < -kStep) dq = -kStep;
        rc->qp_p += dq;
        if (rc->qp_p < rc->qpmin) rc->qp_p = rc->qpmin;
        if (rc->qp_p > rc->qpmax) rc->qp_p = rc->qpmax;
    }
    rc->fill += bits - (double)rc->bitrate / rc->fps;
    if (rc->fill < 0.0) rc->fill = 0.0;
    if (rc->fill > rc->bufbits * 2.0) rc->fill = rc->bufbits * 2.0;
}

void fdv_rc_skip(fdv_rc *rc, size_t bytes) {
    rc->fill += (double)bytes * 8.0 - (double)rc->bitrate / rc->fps;
    if (rc->fill < 0.0) rc->fill = 0.0;
    if (rc->fill > rc->bufbits * 2.0) rc->fill = rc->bufbits * 2.0;
}

}  // extern "C"
