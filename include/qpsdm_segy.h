/*
 * qpsdm_segy.h -- SU trace records and their I/O, drop-in for the reference's
 * segy API (src/segy.h:78-112: fgettr, fputtr, sgettr, sputtr, swaptr).
 *
 * struct segy is the SU trace: the 240-byte SEG-Y trace header in the
 * standard SU field order (the on-disk format every SU file shares; the
 * reference's src/segy.h:123-610 declares the same fields in the same
 * places) followed by up to SU_NFLTS samples.  Files are big-endian; the
 * readers turn the header fields the reference's build selects (its
 * SEGY_<FIELD> switches, src/segy.h:22-65) and the samples into native
 * order and leave the other header bytes as they are on disk; the writers
 * turn those fields and the samples back and write zeros in the other
 * header fields, as the reference's writers do.
 *
 * C++ linkage, as the reference's declarations, so that code built against
 * the reference's headers links against this library unchanged.
 * Implementation: q_psdm_b200/pkg/segy.cpp (libqpsdm_pkg.so).
 */
#ifndef QPSDM_SEGY_H_
#define QPSDM_SEGY_H_

#include <stdio.h>

#define SU_NFLTS 65535 /* samples a trace record can hold */

typedef struct segy segy;

struct segy {
  int tracl, tracr, fldr, tracf, ep, cdp, cdpt; /* bytes 0-27 */
  short trid, nvs, nhs, duse;                    /* 28-35 */
  int offset, gelev, selev, sdepth, gdel, sdel, swdep, gwdep; /* 36-67 */
  short scalel, scalco;                          /* 68-71 */
  int sx, sy, gx, gy;                            /* 72-87 */
  short counit, wevel, swevel, sut, gut, sstat, gstat, tstat, laga, lagb, delrt, muts,
      mute;                                      /* 88-113 */
  unsigned short ns, dt;                         /* 114-117 */
  short gain, igc, igi, corr, sfs, sfe, slen, styp, stas, stae, tatyp, afilf, afils,
      nofilf, nofils, lcf, hcf, lcs, hcs, year, day, hour, minute, sec, timbas, trwf,
      grnors, grnofr, grnlof, gaps, otrav;        /* 118-179 */
  int cdpx, cdpy, iline, xline, sp, unscale, ntr; /* 180-207 */
  short mark, shortpad;                          /* 208-211 */
  short unass[14];                               /* 212-239 */
  float data[SU_NFLTS];
};

/* Next trace of an SU file: header and ns samples; returns ns, 0 at the end
 * of the file or on a short record (src/segy.cc:4480-5119). */
int fgettr(FILE *fp, segy *tr);
/* Appends one trace record (240 + 4 ns bytes) (src/segy.cc:5121-5756). */
void fputtr(FILE *fp, const segy *tr);
/* One trace record from memory (src/segy.cc:6395-7042); returns ns. */
int sgettr(unsigned char *buf, segy *tr);
/* One trace record into memory (src/segy.cc:5758-6393). */
void sputtr(unsigned char *buf, const segy *tr);

#define fvgettr(fp, tr) fgettr(fp, tr)
#define fvputtr(fp, tr) fputtr(fp, tr)
#define swaptr(buf, tr) sgettr(buf, tr)

#endif /* QPSDM_SEGY_H_ */
