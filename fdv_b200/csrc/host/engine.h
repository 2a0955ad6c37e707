// The GPU engine's host-side interface (implemented in device/engine.cu).
#pragma once
#include <cstdint>

#include "fdvb_internal.h"

struct fdvb_engine;

extern "C" {
fdvb_engine *fdvb_engine_create(int nunits, const int *w, const int *h, int range, int device);
void fdvb_engine_destroy(fdvb_engine *E);
int fdvb_engine_units(const fdvb_engine *E);
int fdvb_engine_step(fdvb_engine *E, const uint8_t *const *planes, const int *is_intra, const int *qp,
                     const double *lscale, const int *force_skip);
int fdvb_engine_submit(fdvb_engine *E, const uint8_t *const *planes, const int *is_intra, const int *qp,
                       const double *lscale, const int *force_skip);
int fdvb_engine_collect(fdvb_engine *E);
int fdvb_engine_submit_batch(fdvb_engine *E, int K, const uint8_t *const *planes, const int *is_intra, const int *qp,
                             const double *lscale, const int *force_skip);
int fdvb_engine_max_batch(const fdvb_engine *E);
int fdvb_engine_set_tuning(fdvb_engine *E, int max_batch, int p_grid);
int fdvb_engine_key_lookahead(fdvb_engine *E, const uint8_t *const *planes, const int *qp);
void fdvb_engine_get_tuning(const fdvb_engine *E, int *max_batch, int *p_grid, int *nsm);
void fdvb_engine_defer_refs(fdvb_engine *E, int on);
int fdvb_engine_commit_refs(fdvb_engine *E);
const fdvb_streams *fdvb_engine_pstreams(fdvb_engine *E, int unit);
const fdvb_streams *fdvb_engine_istreams(fdvb_engine *E, int unit, int plane);
int fdvb_engine_recon(fdvb_engine *E, int unit, uint8_t *i420);
int fdvb_engine_set_refs(fdvb_engine *E, int unit, const uint8_t *near_i420, const uint8_t *far_i420);
const char *fdvb_engine_error(void);
void fdvb_engine_src_on_device(fdvb_engine *E, int on);
void fdvb_engine_direct_upload(fdvb_engine *E, int on);
void fdvb_engine_stream_frames(fdvb_engine *E, int on);
int fdvb_engine_ready(fdvb_engine *E);
void fdvb_engine_stats(const fdvb_engine *E, double *step_ms, double *pk_ms, long long *pk_n, double *ik_ms,
                       long long *ik_n, long long *launches, long long *steps, long long *d2h_bytes);
void fdvb_engine_stats_reset(fdvb_engine *E);
void fdvb_engine_set_wait_ns(fdvb_engine *E, unsigned long long ns);
void fdvb_engine_inject_stall(fdvb_engine *E, int unit, int row);
int fdvb_engine_profile(fdvb_engine *E, int enable, unsigned long long *out32);
int fdvb_engine_timeline(fdvb_engine *E, int u, unsigned long long *out);
int fdvb_engine_set_learned(fdvb_engine *E, const float *params, float conf);
int fdvb_engine_records(fdvb_engine *E, int enable);
int fdvb_engine_learned_conf(fdvb_engine *E, const float *conf5);
int fdvb_engine_mb_records(fdvb_engine *E, int unit, uint8_t *mode, int16_t *mv, uint8_t *ref, float *cost);
}
