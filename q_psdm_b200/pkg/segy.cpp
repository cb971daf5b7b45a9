// segy.cpp -- SU trace records, big-endian on disk (include/qpsdm_segy.h).
//
// A table of the header fields the reader and writer convert (offset, width)
// replaces field-by-field code: the fields are those the reference's build
// converts (src/segy.h:22-65, SEGY_<FIELD> switches); the reader leaves every
// other header byte as read, the writer writes zeros there (the reference
// writes a record assembled from the converted fields only,
// src/segy.cc:5121-5756).
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "qpsdm_segy.h"

static_assert(sizeof(segy) == 240 + 4 * SU_NFLTS, "SU header is 240 bytes");
static_assert(offsetof(segy, scalco) == 70 && offsetof(segy, sx) == 72 &&
                  offsetof(segy, ns) == 114 && offsetof(segy, cdpx) == 180 &&
                  offsetof(segy, unass) == 212,
              "SU header field offsets");

namespace {

struct Field {
  unsigned short off, bytes;
};
#define F(name) {(unsigned short)offsetof(segy, name), (unsigned short)sizeof(((segy *)0)->name)}
const Field kFields[] = {
    F(tracl), F(tracr),  F(fldr),  F(tracf), F(ep),     F(cdp),   F(cdpt),  F(trid),
    F(nvs),   F(nhs),    F(offset), F(gelev), F(selev), F(sdepth), F(gdel), F(sdel),
    F(scalel), F(scalco), F(sx),   F(sy),    F(gx),     F(gy),    F(counit), F(wevel),
    F(tstat), F(delrt),  F(muts),  F(mute),  F(ns),     F(dt),    F(minute), F(trwf),
    F(cdpx),  F(cdpy),   F(iline), F(xline),
};
#undef F

inline void swap_bytes(unsigned char *p, int n) {
  for (int i = 0, j = n - 1; i < j; ++i, --j) {
    const unsigned char t = p[i];
    p[i] = p[j];
    p[j] = t;
  }
}

// Converts the table's fields of a header in place (either direction).
void swap_fields(unsigned char *h) {
  for (const Field &f : kFields) swap_bytes(h + f.off, f.bytes);
}

// The header as written: the table's fields converted, zeros elsewhere.
void header_out(const segy *tr, unsigned char *h) {
  std::memset(h, 0, 240);
  const unsigned char *src = reinterpret_cast<const unsigned char *>(tr);
  for (const Field &f : kFields) {
    std::memcpy(h + f.off, src + f.off, f.bytes);
    swap_bytes(h + f.off, f.bytes);
  }
}

void samples_swap(float *d, int ns) {
  for (int i = 0; i < ns; ++i) swap_bytes(reinterpret_cast<unsigned char *>(d + i), 4);
}

}  // namespace

int fgettr(FILE *fp, segy *tr) {
  unsigned char *h = reinterpret_cast<unsigned char *>(tr);
  if (std::fread(h, 240, 1, fp) != 1) return 0;
  swap_fields(h);
  const int ns = tr->ns;
  if ((int)std::fread(tr->data, sizeof(float), ns, fp) != ns) return 0;
  samples_swap(tr->data, ns);
  return ns;
}

int sgettr(unsigned char *buf, segy *tr) {
  unsigned char *h = reinterpret_cast<unsigned char *>(tr);
  std::memcpy(h, buf, 240);
  swap_fields(h);
  const int ns = tr->ns;
  std::memcpy(tr->data, buf + 240, sizeof(float) * ns);
  samples_swap(tr->data, ns);
  return ns;
}

void sputtr(unsigned char *buf, const segy *tr) {
  const int ns = tr->ns;
  header_out(tr, buf);
  std::memcpy(buf + 240, tr->data, sizeof(float) * ns);
  samples_swap(reinterpret_cast<float *>(buf + 240), ns);
}

void fputtr(FILE *fp, const segy *tr) {
  const int ns = tr->ns;
  unsigned char h[240];
  header_out(tr, h);
  std::fwrite(h, 240, 1, fp);
  float chunk[1024];
  for (int i = 0; i < ns; i += 1024) {
    const int n = ns - i < 1024 ? ns - i : 1024;
    std::memcpy(chunk, tr->data + i, sizeof(float) * n);
    samples_swap(chunk, n);
    std::fwrite(chunk, sizeof(float), n, fp);
  }
}
