// Host-side argument validation and kernel-parameter building shared by the
// 2-D and 3-D entry points.
#pragma once

#include <cstring>

#include "dn_common.cuh"

namespace dn {

inline bool box_ok(const dn_box& b, int D, int H, int W) {
  const int n[3] = {D, H, W};
  for (int a = 0; a < 3; ++a)
    if (b.lo[a] < 0 || b.hi[a] > n[a] || b.lo[a] >= b.hi[a]) return false;
  return true;
}

inline BoxDev to_dev(const dn_box& b) {
  BoxDev d;
  for (int a = 0; a < 3; ++a) {
    d.lo[a] = b.lo[a];
    d.hi[a] = b.hi[a];
  }
  return d;
}

// Components used by a solver: 2-D TM {Ez,Hx,Hy}, 2-D TE {Hz,Ex,Ey}, 3-D all.
inline unsigned used_mask(bool is3d, int pol) {
  if (is3d) return 0x3f;
  return pol == DN_TM ? ((1u << DN_EZ) | (1u << DN_HX) | (1u << DN_HY))
                      : ((1u << DN_HZ) | (1u << DN_EX) | (1u << DN_EY));
}

template <typename T>
int build_params(bool is3d, const dn_grid* g, void* const fa[6], void* const fb[6],
                 const void* ce, const dn_cpml* cpml, const dn_source* src,
                 const dn_monitor* mons, int32_t n_mon, const dn_probe* probe, int32_t* status,
                 StepParams<T>* p) {
  if (!g || !fa || !fb || !ce || !cpml) return DN_EINVAL;
  if (g->D < 1 || g->H < 1 || g->W < 1) return DN_EINVAL;
  if (!is3d && g->D != 1) return DN_EINVAL;
  if (g->pitch_y < g->W) return DN_EINVAL;
  if (is3d && g->pitch_z < (int64_t)g->H * g->pitch_y) return DN_EINVAL;
  if (!(g->dt > 0.0) || !(g->dl > 0.0)) return DN_EINVAL;
  if (!is3d && g->pol != DN_TM && g->pol != DN_TE) return DN_EINVAL;
  if (is3d && g->axes != DN_AXES_REFERENCE && g->axes != DN_AXES_PHYSICAL) return DN_EINVAL;
  if (is3d && g->axes == DN_AXES_REFERENCE && !(g->D == g->H && g->H == g->W))
    return DN_EINVAL;  // the reference's broadcasting only exists on cubic grids
  if (n_mon < 0 || n_mon > DN_MAX_MONITORS || (n_mon > 0 && !mons)) return DN_EINVAL;

  std::memset(p, 0, sizeof(*p));
  p->D = g->D;
  p->H = g->H;
  p->W = g->W;
  p->py = g->pitch_y;
  p->pz = is3d ? g->pitch_z : 0;
  const unsigned used = used_mask(is3d, g->pol);
  for (int c = 0; c < 6; ++c) {
    if ((used >> c) & 1u) {
      if (!fa[c] || !fb[c]) return DN_EINVAL;
    }
  }
  p->ce = static_cast<const T*>(ce);
  for (int a = 0; a < 3; ++a) {
    const bool need = is3d ? (a != 0 || g->axes == DN_AXES_PHYSICAL) : (a != 0);
    if (need && (!cpml->b[a] || !cpml->c[a])) return DN_EINVAL;
    p->b[a] = cpml->b[a];
    p->c[a] = cpml->c[a];
  }
  p->dt = static_cast<T>(g->dt);
  p->inv_dl = static_cast<T>(1.0 / g->dl);
  p->src.comp = DN_NONE;
  if (src && src->component != DN_NONE) {
    if (src->component < 0 || src->component > 5) return DN_EINVAL;
    if (!((used >> src->component) & 1u)) return DN_EINVAL;
    if (!box_ok(src->box, g->D, g->H, g->W) || !src->wave) return DN_EINVAL;
    p->src.comp = src->component;
    p->src.box = to_dev(src->box);
    p->src.wave = static_cast<const T*>(src->wave);
  }
  p->n_mon = n_mon;
  for (int m = 0; m < n_mon; ++m) {
    const dn_monitor& M = mons[m];
    if (M.component < 0 || M.component > 5 || !((used >> M.component) & 1u)) return DN_EINVAL;
    if (!box_ok(M.box, g->D, g->H, g->W)) return DN_EINVAL;
    if (M.n_freq < 1 || M.n_freq > DN_MAX_FREQS || !M.phase || !M.acc) return DN_EINVAL;
    p->mon[m].comp = M.component;
    p->mon[m].nf = M.n_freq;
    p->mon[m].box = to_dev(M.box);
    p->mon[m].ncell = p->mon[m].box.cells();
    p->mon[m].phase = M.phase;
    p->mon[m].acc = M.acc;
  }
  p->probe.comp = DN_NONE;
  if (probe && probe->component != DN_NONE) {
    if (probe->component < 0 || probe->component > 5 || !((used >> probe->component) & 1u))
      return DN_EINVAL;
    const int n[3] = {g->D, g->H, g->W};
    for (int a = 0; a < 3; ++a)
      if (probe->pos[a] < 0 || probe->pos[a] >= n[a]) return DN_EINVAL;
    if (!probe->out) return DN_EINVAL;
    p->probe.comp = probe->component;
    for (int a = 0; a < 3; ++a) p->probe.pos[a] = probe->pos[a];
    p->probe.out = static_cast<T*>(probe->out);
  }
  p->status = status;
  return DN_OK;
}

// The source waveform, the monitor phase tables and the probe output are
// indexed by the absolute step and carry their length (n_t).  A run or a
// reverse sweep over steps [t_lo, t_hi) may only touch rows below n_t; this is
// checked before anything is queued, so a too-long call returns DN_EINVAL
// instead of reading or writing past the caller's arrays.
inline bool mons_steps_ok(const dn_monitor* mons, int32_t n_mon, int64_t t_lo, int64_t t_hi) {
  if (t_lo < 0 || t_hi < t_lo) return false;
  for (int m = 0; m < n_mon; ++m)
    if (mons[m].n_t < 0 || t_hi > mons[m].n_t) return false;
  return true;
}

inline bool steps_ok(const dn_source* src, const dn_monitor* mons, int32_t n_mon,
                     const dn_probe* probe, int64_t t_lo, int64_t t_hi) {
  if (!mons_steps_ok(mons, n_mon, t_lo, t_hi)) return false;
  if (src && src->component != DN_NONE && t_hi > src->n_t) return false;
  if (probe && probe->component != DN_NONE && t_hi > probe->n_t) return false;
  return true;
}

template <typename T>
void set_io(StepParams<T>* p, void* const from[6], void* const to[6]) {
  for (int c = 0; c < 6; ++c) {
    p->in[c] = static_cast<const T*>(from[c]);
    p->out[c] = static_cast<T*>(to[c]);
  }
}

}  // namespace dn
