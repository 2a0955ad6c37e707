// Device-side descriptors of the batched encoder engine.
#pragma once
#include "common.cuh"
#include "learned.cuh"

namespace fdvb {

// One encoder unit (a horizontal band of a stream, or a whole stream) as the
// analysis kernels see it for the current frame.
struct UnitDev {
    int w, h, mbw, mbh;
    const uint8_t *cur[3];      // source planes, tight
    uint8_t *rec[3];            // reconstruction, tight
    RefPlanes ref[2];           // nearest, and second (== nearest when only one is valid)
    MBInfo *mbi;                // per macroblock, this frame
    int *progress;              // per macroblock row: a 64-bit progress word (pframe.cuh), 8-byte aligned
    uint8_t *slots;             // per macroblock symbol slot (P-frames)
    double lambda;
    int qp, navail, force_skip, range;
    int stall_row;              // test hook: this row never runs (-1: none)
    unsigned long long *prof;   // optional per-phase cycle accumulators (NULL: off)
    const lrn::Hint *hint;      // learned proposals per macroblock (NULL: the plain search)
    double skip_gate;           // a confident SKIP needs its RD cost <= skip_gate * lambda (<= 0: no gate)
    int inter8;                 // the confident-inter path also tries INTER8 (seeded, short searches)
    float *mbcost;              // per macroblock: RD cost of the chosen mode (NULL: off)
    // per macroblock, from lrn_preskip_kernel (NULL: none): the RD cost of a
    // confident SKIP with the zero vector that passed the gate, its
    // reconstruction already written; -1 otherwise
    const float *prejs;
    // per macroblock, with the phase profile on (NULL: off): %globaltimer when
    // its wait for the row above ended and when it published its progress
    unsigned long long *tl;
    // The reference this frame becomes (post.cuh), written tile by tile as
    // the wavefront passes, and per macroblock row the count of tiles written
    // (NULL: no post stage; the deblock and reference-preparation kernels run
    // after the frame instead).
    OutPlanes out;
    int *post_prog;
    // The previous frame's tile counts when that frame is still being coded
    // by the same launch (its output is this frame's nearest reference): each
    // macroblock waits for the tiles its reference reads reach (NULL: the
    // references are complete).
    const int *ref_prog;
    // The learned inference's reference luma (stride lrs) when it is not the
    // nearest reference: frames after the first of a batched launch use the
    // previous frame's source (their reference does not exist before the
    // launch).  NULL: ref[0].G.
    const uint8_t *lref;
    int lrs;
};

// Phases of a macroblock, for the optional cycle profile.
enum { PP_WAIT = 0, PP_LOAD, PP_SKIP, PP_SEARCH, PP_RESID, PP_DECIDE, PP_COMMIT, PP_OUT, PP_NMB, PP_NSKIP,
       PP_G0, PP_G1, PP_G2, PP_G3, PP_IT16, PP_IT8, PP_N = 16 };

struct RowTask { int unit, row; };

// Stream ids of the P-frame slot (fdv.h:4170, :6198-6210).
enum { PS_REF = 4, PS_MVX = 5, PS_MVY = 6, PS_SUB = 7, PS_MERGE = 8, PS_CN = 9 };

// One frame of a P launch whose frames are compacted inside the launch: the
// block that finishes a unit's last macroblock row of the frame compacts that
// unit's symbol streams, and the last unit of the frame to be compacted sets
// the frame's host-mapped word, so the host can code the frame while the
// launch goes on.
struct FrameSync {
    unsigned *ready;       // host-mapped; set to ready_val once the frame's streams are in place
    unsigned ready_val;
};

}  // namespace fdvb
