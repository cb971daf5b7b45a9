/*
 * physics_fp32.c -- FP32 restatement of the engine's plain physics kernel.
 *
 * TEST INFRASTRUCTURE ONLY (tests/, bench.py's cpu_baseline leg).
 *
 * The reference's image_depth_gpu (src/q-psdm.cu:2246-2379) stubs its
 * traveltimes (ts = tg = 1, :2350-2351), so the physics method has no
 * runnable reference; physics_oracle.c states it in FP64.  This file
 * restates, operation by operation, the FP32 arithmetic of the engine's
 * plain physics kernel (q_psdm_b200/csrc/physics.cu, k_image_plain with FP32
 * panels), so that -- given the same panels, tables, dips and gate results --
 * it computes the same image bit for bit: the integer picks (it1, the t*
 * bin b0), the dip mask and the point-trace count pinned exactly, the way
 * the compat path is pinned against the reference's own kernel.
 *
 * Rules that make the bits agree: one IEEE rounding per operation (built
 * with -ffp-contract=off), fused multiply-adds only where the kernel writes
 * them (fmaf, correctly rounded), correctly rounded division and sqrtf,
 * truncating float->int conversion, and each point summing its traces in
 * submission order.  Per point (the kernel's thread):
 *
 *   cell / depth node as src/q-psdm.cu:2343-2349; t, t* of source and
 *   receiver bilinear in surface position, linear in depth; dip test and
 *   taper (:2303-2340); it1 = (int)(t / dt1), t* bin; amplitude weight
 *   v (r + 1/r) (:2366-2374); sample linear in time and t*.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

typedef struct {
  int64_t idx;
  uint16_t nys, nxs, dys, dxs;
} f32_desc;

typedef struct {
  int nzi, nxb, ixstart, nt, nbins;
  float dt1, dxi, dzi, taperzone, dtstar, dzii;
  int tcdp1, tcdp2; /* relative to fci */
  int nxg, nzg, nxi1, nzi1;
} orc_p32;

static inline float lerpf(float a, float b, float w) { return fmaf(w, b - a, a); }

static inline float bilinf(const float *tab, int64_t base, int64_t sx, int64_t sy, float wx,
                           float wy) {
  return lerpf(lerpf(tab[base], tab[base + sx], wx),
               lerpf(tab[base + sy], tab[base + sy + sx], wx), wy);
}

static inline int grid_pos(float px, float py, float xc, float rdx, float rdy, float hx,
                           float hy, int nxs, int nys, float *fx, float *fy) {
  *fx = fmaf(px - xc, rdx, hx);
  *fy = fmaf(py, rdy, hy);
  return *fx >= 0.0f && *fx <= (float)(nxs - 1) && *fy >= 0.0f && *fy <= (float)(nys - 1);
}

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

static int table_node(const f32_desc *d, const float *tab, float px, float py, float xc,
                      int poff, int nxi1, int nzi1, float *v) {
  const int nxs = d->nxs, nys = d->nys;
  float fx, fy;
  if (!grid_pos(px, py, xc, 1.0f / (float)d->dxs, 1.0f / (float)d->dys,
                0.5f * (float)(nxs - 1), 0.5f * (float)(nys - 1), nxs, nys, &fx, &fy))
    return 0;
  const int ix = imin((int)fx, imax(nxs - 2, 0)), iy = imin((int)fy, imax(nys - 2, 0));
  const float wx = nxs > 1 ? fx - (float)ix : 0.0f, wy = nys > 1 ? fy - (float)iy : 0.0f;
  const int64_t sx = nxs > 1 ? (int64_t)nxi1 * nzi1 : 0;
  const int64_t sy = nys > 1 ? (int64_t)nxs * nxi1 * nzi1 : 0;
  const int64_t base = d->idx + (int64_t)(iy * nxs + ix) * nxi1 * nzi1 + poff;
  *v = bilinf(tab, base, sx, sy, wx, wy);
  return 1;
}

typedef struct {
  int ok, same, offA, offB, nxs, nys;
  float c2, xc, rdx, rdy, hx, hy;
  const f32_desc *tA, *tB, *qA, *qB;
} cells32;

static int same_grid(const f32_desc *a, const f32_desc *b) {
  return a->nxs == b->nxs && a->nys == b->nys && a->dxs == b->dxs && a->dys == b->dys;
}

static void setup_cells(cells32 *pc, int ixi, float z, const orc_p32 *a, const f32_desc *dt,
                        const f32_desc *dq) {
  pc->ok = 0;
  pc->same = 0;
  if (ixi < a->tcdp1 || ixi > a->tcdp2) return;
  const int lx = ixi - a->tcdp1;
  const int ixg = lx / a->nxi1;
  const int ixl = lx - ixg * a->nxi1;
  const float fz = z / a->dzii;
  const int izn = (int)fz;
  pc->c2 = fz - (float)izn;
  int izgA = izn / a->nzi1, izgB = (izn + 1) / a->nzi1;
  int izlA = izn - izgA * a->nzi1;
  int izlB = izn + 1 - izgB * a->nzi1;
  if (izgB >= a->nzg) {
    izgB = izgA;
    izlB = izlA;
    pc->c2 = 0.0f;
  }
  if (ixg >= a->nxg || izgA >= a->nzg) return;
  pc->ok = 1;
  pc->offA = ixl * a->nzi1 + izlA; /* reference layout [ixl][izl] */
  pc->offB = ixl * a->nzi1 + izlB;
  const int cA = ixg * a->nzg + izgA, cB = ixg * a->nzg + izgB;
  pc->tA = dt + cA;
  pc->tB = dt + cB;
  pc->qA = dq + cA;
  pc->qB = dq + cB;
  pc->xc = ((float)(a->tcdp1 + ixg * a->nxi1) + 0.5f * (float)(a->nxi1 - 1)) * a->dxi;
  pc->same = same_grid(pc->tA, pc->tB) && same_grid(pc->tA, pc->qA) &&
             same_grid(pc->tA, pc->qB);
  pc->nxs = pc->tA->nxs;
  pc->nys = pc->tA->nys;
  pc->rdx = 1.0f / (float)pc->tA->dxs;
  pc->rdy = 1.0f / (float)pc->tA->dys;
  pc->hx = 0.5f * (float)(pc->tA->nxs - 1);
  pc->hy = 0.5f * (float)(pc->tA->nys - 1);
}

static int lookup_tq(const cells32 *pc, const float *ttt, const float *qqq, int nxi1, int nzi1,
                     float px, float py, float *t, float *q) {
  if (pc->same) {
    const int nxs = pc->nxs, nys = pc->nys;
    float fx, fy;
    if (!grid_pos(px, py, pc->xc, pc->rdx, pc->rdy, pc->hx, pc->hy, nxs, nys, &fx, &fy))
      return 0;
    const int ix = imin((int)fx, imax(nxs - 2, 0)), iy = imin((int)fy, imax(nys - 2, 0));
    const float wx = nxs > 1 ? fx - (float)ix : 0.0f, wy = nys > 1 ? fy - (float)iy : 0.0f;
    const int64_t plane = (int64_t)nxi1 * nzi1;
    const int64_t sx = nxs > 1 ? plane : 0, sy = nys > 1 ? (int64_t)nxs * plane : 0;
    const int64_t off = (int64_t)(iy * nxs + ix) * plane;
    const float ta = bilinf(ttt, pc->tA->idx + off + pc->offA, sx, sy, wx, wy);
    const float tb = bilinf(ttt, pc->tB->idx + off + pc->offB, sx, sy, wx, wy);
    const float qa = bilinf(qqq, pc->qA->idx + off + pc->offA, sx, sy, wx, wy);
    const float qb = bilinf(qqq, pc->qB->idx + off + pc->offB, sx, sy, wx, wy);
    *t = lerpf(ta, tb, pc->c2);
    *q = lerpf(qa, qb, pc->c2);
    return 1;
  }
  float ta, tb, qa, qb;
  if (!table_node(pc->tA, ttt, px, py, pc->xc, pc->offA, nxi1, nzi1, &ta)) return 0;
  if (!table_node(pc->tB, ttt, px, py, pc->xc, pc->offB, nxi1, nzi1, &tb)) return 0;
  if (!table_node(pc->qA, qqq, px, py, pc->xc, pc->offA, nxi1, nzi1, &qa)) return 0;
  if (!table_node(pc->qB, qqq, px, py, pc->xc, pc->offB, nxi1, nzi1, &qb)) return 0;
  *t = lerpf(ta, tb, pc->c2);
  *q = lerpf(qa, qb, pc->c2);
  return 1;
}

/* ints: [ntr][8] gate results (status 3 = accepted; ixi1 at 4, ixi2 at 5,
 * izimin at 7); geom: [ntr][4] (sx, sy, gx, gy relative); panels: FP32
 * [ntr][nbins][nt] (the engine's panels of those traces); dips: 4 x
 * [nxi][nzi]; img: [nxb][nzi] float, accumulated in place; counts[0] +=
 * point-traces, counts[1] += imaged pairs. */
void orc_image_plain_fp32(const orc_p32 *a, int ntr, const int *ints, const float *geom,
                          const float *panels, const float *dips, size_t nxz,
                          const f32_desc *dt, const float *ttt, const f32_desc *dq,
                          const float *qqq, float *img, long long *counts) {
  long long npt = 0, nimg = 0;
  const size_t pstride = (size_t)a->nbins * a->nt;
  const float inv_dt1 = 1.0f / a->dt1, inv_dts = 1.0f / a->dtstar;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : npt, nimg)
  for (long long pt = 0; pt < (long long)a->nxb * a->nzi; ++pt) {
    const int ixb = (int)(pt / a->nzi), izi = (int)(pt % a->nzi);
    const int ixi = ixb + a->ixstart;
    const float z = (float)izi * a->dzi;
    const size_t k = (size_t)ixi * a->nzi + izi;
    const float tanx1 = dips[k], tanx2 = dips[nxz + k];
    const float tany1 = dips[2 * nxz + k], tany2 = dips[3 * nxz + k];
    cells32 pc;
    setup_cells(&pc, ixi, z, a, dt, dq);
    if (!pc.ok) continue;
    const float tz = a->taperzone;
    const float tanx1c = tanx1 - tz * fmaf(tanx1, tanx1, 1.0f);
    const float tanx2c = tanx2 + tz * fmaf(tanx2, tanx2, 1.0f);
    const float tany1c = tany1 - tz * fmaf(tany1, tany1, 1.0f);
    const float tany2c = tany2 + tz * fmaf(tany2, tany2, 1.0f);
    const float z2 = z * z;
    const float x = (float)ixi * a->dxi;
    float acc = img[(size_t)ixb * a->nzi + izi];
    for (int i = 0; i < ntr; ++i) {
      const int *q = ints + (size_t)i * 8;
      if (q[0] != 3 || ixi < q[4] || ixi > q[5] || izi < q[7]) continue;
      const float *gm = geom + (size_t)i * 4;
      float ts, qs, tg, qg;
      if (!lookup_tq(&pc, ttt, qqq, a->nxi1, a->nzi1, gm[0], gm[1], &ts, &qs)) continue;
      if (!lookup_tq(&pc, ttt, qqq, a->nxi1, a->nzi1, gm[2], gm[3], &tg, &qg)) continue;
      ++npt;
      const float dsx = gm[0] - x, dgx = gm[2] - x;
      const float ds = sqrtf(fmaf(dsx, dsx, fmaf(gm[1], gm[1], z2)));
      const float dg = sqrtf(fmaf(dgx, dgx, fmaf(gm[3], gm[3], z2)));
      const float rs = 1.0f / ds, rg2 = 1.0f / dg;
      const float ux = fmaf(dsx, rs, dgx * rg2);
      const float uy = fmaf(gm[1], rs, gm[3] * rg2);
      const float uz = z * (rs + rg2);
      const float tanx = ux / uz, tany = uy / uz;
      if (!(tanx > tanx1c && tanx < tanx2c && tany > tany1c && tany < tany2c)) continue;
      float w = 1.0f;
      if (tanx < tanx1) w = w * ((tanx - tanx1c) / (tanx1 - tanx1c));
      if (tanx > tanx2) w = w * ((tanx2c - tanx) / (tanx2c - tanx2));
      if (tany < tany1) w = w * ((tany - tany1c) / (tany1 - tany1c));
      if (tany > tany2) w = w * ((tany2c - tany) / (tany2c - tany2));
      const float t = ts + tg;
      const float ft = t * inv_dt1;
      const int it1 = (int)ft;
      if (!(it1 > 0 && it1 + 1 < a->nt)) continue;
      ++nimg;
      const float wt = ft - (float)it1;
      const float fb = fminf(fmaxf((qs + qg) * inv_dts, 0.0f), (float)(a->nbins - 1));
      const int b0 = imin((int)fb, a->nbins - 2);
      const float wb = fb - (float)b0;
      const float *pp = panels + (size_t)i * pstride + (size_t)b0 * a->nt + it1;
      const float smp = lerpf(lerpf(pp[0], pp[1], wt), lerpf(pp[a->nt], pp[a->nt + 1], wt), wb);
      const float v = t > 0.1f ? 100.0f / (t * t) : 10000.0f;
      const float dr = ds * rg2;
      const float r = ((dr * dr) * dr) * (tg / ts);
      const float val = ((w * (r + 1.0f / r)) * v) * smp;
      acc = acc + val;
    }
    img[(size_t)ixb * a->nzi + izi] = acc;
  }
  if (counts) {
    counts[0] += npt;
    counts[1] += nimg;
  }
}
