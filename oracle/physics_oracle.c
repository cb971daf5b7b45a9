/*
 * physics_oracle.c -- FP64 oracle of the physics imaging mode.
 *
 * TEST INFRASTRUCTURE ONLY (tests/, smoke(), bench.py cpu_baseline).
 *
 * The reference's image_depth_gpu (src/q-psdm.cu:2246-2379) receives the
 * traveltime and t* tables, the spectra and the gain-limit constants but
 * stubs the imaging (ts = tg = 1, :2350-2351), so physics mode has no
 * runnable reference: parity is unpinned by the reference and is stated
 * against this double-precision restatement of the method:
 *
 *   for every image point (x, z) of the block and every accepted trace whose
 *   column range holds x and whose source and receiver both lie inside the
 *   surface grid of the point's table cells (a point-trace):
 *     ts, t*s, tg, t*g  from the tables: cell (ixg, izg) of the point, the
 *                       cell's surface grid centred on the cell (bilinear in
 *                       surface position), linear between depth nodes
 *                       (src/q-psdm.cu:2343-2349 gives the cell mapping)
 *     t = ts + tg, t* = t*s + t*g
 *     sample = linear in time on the dt1 grid between the two t* panels
 *              around t*  (panels: compensated traces, computed in numpy
 *              float64 by oracle.physics_panels)
 *     dip taper w and amplitude weight as src/q-psdm.cu:2303-2378
 *     img += w * (r + 1/r) * v * sample      (all in double)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

typedef struct {
  int64_t idx;
  uint16_t nys, nxs, dys, dxs;
} orc_desc;

typedef struct {
  int nzi, nxb, ixstart, nt, nbins;
  double dt1, dxi, dzi, taperzone, dtstar, dzii;
  int tcdp1, tcdp2; /* relative to fci */
  int nxg, nzg, nxi1, nzi1;
} orc_phys_params;

/* The surface-grid test of a lookup, in the engine's FP32 arithmetic (one
 * rounding per operation, the fused multiply-add as fmaf), so that a pair is
 * evaluated -- and counted -- exactly when the engine evaluates it:
 * fx = fma(px - xc, 1/dxs, (nxs-1)/2) inside [0, nxs-1], fy likewise. */
static int in_grid(const orc_desc *d, float px, float py, float xc) {
  const float rdx = 1.0f / (float)d->dxs, rdy = 1.0f / (float)d->dys;
  const float fx = fmaf(px - xc, rdx, 0.5f * (float)(d->nxs - 1));
  const float fy = fmaf(py, rdy, 0.5f * (float)(d->nys - 1));
  return fx >= 0.0f && fx <= (float)(d->nxs - 1) && fy >= 0.0f && fy <= (float)(d->nys - 1);
}

/* value at one depth node of one cell for surface point (px, py) */
static int tab_node(const orc_desc *d, const float *tab, float pxf, float pyf,
                    float xcf, int ixl, int izl, int nxi1, int nzi1,
                    double *v) {
  if (!in_grid(d, pxf, pyf, xcf)) return 0;
  const double px = pxf, py = pyf, xc = xcf;
  int nxs = d->nxs, nys = d->nys;
  double fx = (px - xc) / d->dxs + 0.5 * (nxs - 1);
  double fy = py / d->dys + 0.5 * (nys - 1);
  if (fx < 0.0) fx = 0.0;
  if (fx > nxs - 1) fx = nxs - 1;
  if (fy < 0.0) fy = 0.0;
  if (fy > nys - 1) fy = nys - 1;
  int ix = (int)fx, iy = (int)fy;
  if (ix > nxs - 2) ix = nxs - 2 < 0 ? 0 : nxs - 2;
  if (iy > nys - 2) iy = nys - 2 < 0 ? 0 : nys - 2;
  double wx = nxs > 1 ? fx - ix : 0.0, wy = nys > 1 ? fy - iy : 0.0;
  int64_t sx = nxs > 1 ? (int64_t)nxi1 * nzi1 : 0;
  int64_t sy = nys > 1 ? (int64_t)nxs * nxi1 * nzi1 : 0;
  int64_t b = d->idx + ((int64_t)(iy * nxs + ix) * nxi1 + ixl) * nzi1 + izl;
  double v00 = tab[b], v01 = tab[b + sx], v10 = tab[b + sy], v11 = tab[b + sy + sx];
  *v = (1 - wy) * ((1 - wx) * v00 + wx * v01) + wy * ((1 - wx) * v10 + wx * v11);
  return 1;
}

typedef struct {
  int ok, ixl, izlA, izlB;
  double c2;
  float xc; /* the cell's centre x in the engine's FP32 arithmetic */
  const orc_desc *tA, *tB, *qA, *qB;
} cells_t;

static int lookup(const cells_t *c, const float *ttt, const float *qqq, int nxi1,
                  int nzi1, float px, float py, double *t, double *q) {
  double ta, tb, qa, qb;
  if (!tab_node(c->tA, ttt, px, py, c->xc, c->ixl, c->izlA, nxi1, nzi1, &ta)) return 0;
  if (!tab_node(c->tB, ttt, px, py, c->xc, c->ixl, c->izlB, nxi1, nzi1, &tb)) return 0;
  if (!tab_node(c->qA, qqq, px, py, c->xc, c->ixl, c->izlA, nxi1, nzi1, &qa)) return 0;
  if (!tab_node(c->qB, qqq, px, py, c->xc, c->ixl, c->izlB, nxi1, nzi1, &qb)) return 0;
  *t = (1 - c->c2) * ta + c->c2 * tb;
  *q = (1 - c->c2) * qa + c->c2 * qb;
  return 1;
}

/* geom: [ntr][4] floats (sx, sy, gx, gy relative); ints3: [ntr][3]
 * (ixi1, ixi2, izimin) of accepted traces; panels: [ntr][nbins][nt] double;
 * img: [nxb][nzi] double, accumulated. */
void orc_physics_image(const orc_phys_params *p, int ntr, const float *geom,
                       const int *ints3, const double *panels,
                       const float *dipx1, const float *dipx2,
                       const float *dipy1, const float *dipy2,
                       const orc_desc *dt, const float *ttt, const orc_desc *dq,
                       const float *qqq, double *img, long long *npt_out) {
  long long npt = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : npt)
  for (int ixb = 0; ixb < p->nxb; ++ixb) {
    int ixi = ixb + p->ixstart;
    for (int izi = 0; izi < p->nzi; ++izi) {
      size_t k = (size_t)ixi * p->nzi + izi;
      double tx1 = dipx1[k], tx2 = dipx2[k], ty1 = dipy1[k], ty2 = dipy2[k];
      double tz = p->taperzone;
      double tx1c = tx1 - tz * (1 + tx1 * tx1), tx2c = tx2 + tz * (1 + tx2 * tx2);
      double ty1c = ty1 - tz * (1 + ty1 * ty1), ty2c = ty2 + tz * (1 + ty2 * ty2);
      double z = izi * p->dzi, x = ixi * p->dxi;
      cells_t c = {0};
      if (ixi >= p->tcdp1 && ixi <= p->tcdp2) {
        int lx = ixi - p->tcdp1, ixg = lx / p->nxi1;
        double fz = z / p->dzii;
        int izn = (int)fz;
        int izgA = izn / p->nzi1, izgB = (izn + 1) / p->nzi1;
        c.ixl = lx - ixg * p->nxi1;
        c.c2 = fz - izn;
        c.izlA = izn - izgA * p->nzi1;
        c.izlB = izn + 1 - izgB * p->nzi1;
        if (izgB >= p->nzg) {
          izgB = izgA;
          c.izlB = c.izlA;
          c.c2 = 0.0;
        }
        if (ixg < p->nxg && izgA < p->nzg) {
          c.ok = 1;
          c.tA = dt + ixg * p->nzg + izgA;
          c.tB = dt + ixg * p->nzg + izgB;
          c.qA = dq + ixg * p->nzg + izgA;
          c.qB = dq + ixg * p->nzg + izgB;
          c.xc = ((float)(p->tcdp1 + ixg * p->nxi1) + 0.5f * (float)(p->nxi1 - 1)) *
                 (float)p->dxi;
        }
      }
      if (!c.ok) continue;
      double acc = 0.0;
      for (int itr = 0; itr < ntr; ++itr) {
        const int *q3 = ints3 + 3 * itr;
        if (ixi < q3[0] || ixi > q3[1] || izi < q3[2]) continue;
        const float *g = geom + 4 * itr;
        double sx = g[0], sy = g[1], gx = g[2], gy = g[3];
        double ts, qs, tg, qg;
        /* a point-trace: inside the trace's aperture, with table values for
         * both its source and its receiver (the pairs the kernel evaluates) */
        if (!lookup(&c, ttt, qqq, p->nxi1, p->nzi1, g[0], g[1], &ts, &qs)) continue;
        if (!lookup(&c, ttt, qqq, p->nxi1, p->nzi1, g[2], g[3], &tg, &qg)) continue;
        ++npt;
        double dsx = sx - x, dgx = gx - x;
        double ds = sqrt(dsx * dsx + sy * sy + z * z);
        double dg = sqrt(dgx * dgx + gy * gy + z * z);
        double ux = dsx / ds + dgx / dg, uy = sy / ds + gy / dg, uz = z / ds + z / dg;
        double tanx = ux / uz, tany = uy / uz;
        if (!(tanx > tx1c && tanx < tx2c && tany > ty1c && tany < ty2c)) continue;
        double w = 1.0;
        if (tanx < tx1) w *= (tanx - tx1c) / (tx1 - tx1c);
        if (tanx > tx2) w *= (tx2c - tanx) / (tx2c - tx2);
        if (tany < ty1) w *= (tany - ty1c) / (ty1 - ty1c);
        if (tany > ty2) w *= (ty2c - tany) / (ty2c - ty2);
        double t = ts + tg;
        double ft = t / p->dt1;
        int it1 = (int)ft;
        if (!(it1 > 0 && it1 + 1 < p->nt)) continue;
        double wt = ft - it1;
        double fb = (qs + qg) / p->dtstar;
        if (fb < 0) fb = 0;
        if (fb > p->nbins - 1) fb = p->nbins - 1;
        int b0 = (int)fb;
        if (b0 > p->nbins - 2) b0 = p->nbins - 2;
        double wb = fb - b0;
        const double *pp = panels + ((size_t)itr * p->nbins + b0) * p->nt + it1;
        double s0 = (1 - wt) * pp[0] + wt * pp[1];
        double s1 = (1 - wt) * pp[p->nt] + wt * pp[p->nt + 1];
        double smp = (1 - wb) * s0 + wb * s1;
        double v = t > 0.1 ? 100.0 / (t * t) : 10000.0;
        double r = ds / dg * ds / dg * ds / dg * tg / ts;
        acc += w * (r + 1.0 / r) * v * smp;
      }
      img[(size_t)ixb * p->nzi + izi] += acc;
    }
  }
  if (npt_out) *npt_out = npt;
}
