/*
 * qpsdm_psdmpkg.h -- the q-psdm driver's utility API, drop-in for the
 * reference's psdmpkg (src/psdmpkg.h:17-213): command-line and par.dat
 * parameters, list and tuple parsers, the end taper of a trace window, the
 * time-offset mute, coordinate scales, 2-D arrays with one contiguous block,
 * project-path parsing and file helpers.  Same names, signatures, linkage
 * and results; the differences, all where the reference fails, are noted
 * at the functions.  Implementation: q_psdm_b200/pkg/psdmpkg.cpp
 * (libqpsdm_pkg.so).
 */
#ifndef QPSDM_PSDMPKG_H_
#define QPSDM_PSDMPKG_H_

#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/stat.h>
#include <unistd.h>

#include "qpsdm_segy.h"

/* The command line given to initargs (src/psdmpkg.cc:3-5). */
extern int xargc;
extern char **xargv;
extern int inited;

/* Arrays: nD arrays are one contiguous block with row pointers, p[0] the
 * block (src/psdmpkg.cc:24-107, :864-977).  Allocation failure prints a
 * message and exits, as the reference.  malloc3i, malloc3f, malloc4f,
 * malloc1d and malloc2d are declared by the reference's header but defined
 * nowhere in it; here they allocate what its free3i/free3f/free4f/free1d/
 * free2d release. */
char *malloc1c(size_t n1);
char **malloc2c(size_t n1, size_t n2);
int *malloc1i(size_t n1);
int **malloc2i(size_t n1, size_t n2);
int ***malloc3i(size_t n1, size_t n2, size_t n3);
float *malloc1f(size_t n1);
float **malloc2f(size_t n1, size_t n2);
float ***malloc3f(size_t n1, size_t n2, size_t n3);
float ****malloc4f(size_t n1, size_t n2, size_t n3, size_t n4);
double *malloc1d(size_t n1);
double **malloc2d(size_t n1, size_t n2);
void free1c(char *p);
void free2c(char **p);
void free1i(int *p);
void free2i(int **p);
void free3i(int ***p);
void free1f(float *p);
void free2f(float **p);
void free3f(float ***p);
void free4f(float ****p);
void free1d(double *p);
void free2d(double **p);

#define alloc1char(n1) malloc1c(n1)
#define alloc2char(n1, n2) malloc2c(n1, n2)
#define alloc1float(n1) malloc1f(n1)
#define alloc1int(n1) malloc1i(n1)
#define alloc2float(n1, n2) malloc2f(n1, n2)
#define alloc2int(n1, n2) malloc2i(n1, n2)
#define free1char(p) free1c(p)
#define free2char(p) free2c(p)
#define free1int(p) free1i(p)
#define free2int(p) free2i(p)
#define free3int(p) free3i(p)
#define free1float(p) free1f(p)
#define free2float(p) free2f(p)
#define free3float(p) free3f(p)
#define free4float(p) free4f(p)
#define free1double(p) free1d(p)
#define free2double(p) free2d(p)

/* "a,b-c,d:s:e" -> the integers it lists, *n of them (malloc'd): ranges
 * b..c, and d, d+s, ... up to e for a stride s of either sign
 * (src/psdmpkg.cc:108-204).  A descending range "c-b" lists nothing where
 * the reference allocates a negative count. */
#define parseline(str, n) parseint(str, n)
int *parseint(const char *str, int *n);

/* The command line: key=value words, the first word with the key wins
 * (src/psdmpkg.cc:7-22, :233-336); 1 when found.  Exit when initargs was
 * not called, as the reference. */
void initargs_inner(int argc, char *argv[], const char *sdoc[]);
int getparint(const char *key, int *val);
int getparfloat(const char *key, float *val);
int getpardouble(const char *key, double *val);
int getparstr(const char *key, char **val);
int getparstr(const char *key, const char **val);
#define getparstring(key, val) getparstr(key, val)

/* Without arguments (and with a terminal on stdin) print the self-doc and
 * exit, as the reference's initargs (src/psdmpkg.h:78-102). */
#define initargs(argc, argv, sdoc)                                   \
  do {                                                               \
    struct stat st_;                                                 \
    if ((argc) == 1 && fstat(fileno(stdin), &st_) == 0 &&            \
        S_ISCHR(st_.st_mode)) {                                      \
      for (int i_ = 0; (sdoc)[i_] != NULL; ++i_)                     \
        fprintf(stderr, "%s", (sdoc)[i_]);                           \
      exit(0);                                                       \
    }                                                                \
    initargs_inner(argc, argv, sdoc);                                \
  } while (0)

#define egetparstring(name, value)                            \
  do {                                                        \
    if (!getparstring(name, value)) {                         \
      fprintf(stderr, "Error: %s must be specified\n", name); \
      exit(0);                                                \
    }                                                         \
  } while (0)
#define egetparint(name, value)                               \
  do {                                                        \
    if (!getparint(name, value)) {                            \
      fprintf(stderr, "Error: %s must be specified\n", name); \
      exit(0);                                                \
    }                                                         \
  } while (0)
#define egetparfloat(name, value)                             \
  do {                                                        \
    if (!getparfloat(name, value)) {                          \
      fprintf(stderr, "Error: %s must be specified\n", name); \
      exit(0);                                                \
    }                                                         \
  } while (0)
#define egetpardouble(name, value)                            \
  do {                                                        \
    if (!getpardouble(name, value)) {                         \
      fprintf(stderr, "Error: %s must be specified\n", name); \
      exit(0);                                                \
    }                                                         \
  } while (0)

/* par.dat records (src/psdmpkg.cc:338-574): fmt is "key=%d,key2=%f,..."
 * with %d, %f/%g, %s (first word) or %S (the rest of the record, malloc'd);
 * '#' starts a comment, a trailing backslash continues a record, blanks
 * around a record are ignored.  Each pattern is matched against every
 * record; matches fill the variadic outputs in the order they are found.
 * Returns the number of matches when every pattern matched exactly once,
 * else -1 (a key given twice: the first record's value has been stored). */
int readparfile(const char *filename, const char *fmt, ...);

/* data[it1..it2] (zero outside [0, ns)) into data1, both ends tapered by
 * 0.5 - 0.5 cos(pi it / 200) over 200 samples (src/psdmpkg.cc:208-231). */
int fetch_and_taper(const float *data, int ns, int it1, int it2, float *data1);

size_t fsize(const char *path);
/* 1 when the file can be read and written (src/psdmpkg.cc:206). */
#define exist(_p) fexist(_p)
int fexist(const char *path);
/* Reverses p in place.  Returns p (the reference returns a pointer to its
 * middle, which no caller uses). */
char *strrev1(char *p);
/* Removes trailing characters c (src/psdmpkg.cc:616-631). */
char *strrtrim(char *src, int c);

/* "<projpath>/<iproc>/<task>" -> its parts; projname the last component of
 * projpath (src/psdmpkg.cc:633-684). */
void parsepath(char *path, char *projpath, char *projname, int *iproc, char *task);

/* "(a,b),(c,d),..." -> *ntuple tuples of *nelem floats (malloc'd), NULL
 * when the brackets or the element counts do not match
 * (src/psdmpkg.cc:686-862).  Differences where the reference fails: one
 * tuple is parsed (the reference writes past an empty allocation and
 * returns NULL), and signs belong to numbers (the reference loops forever
 * on a '-'). */
float *parsetuple(const char *str, int *ntuple, int *nelem);

/* Mute pairs (depth-or-time, offset) made increasing in both
 * (src/psdmpkg.cc:576-599). */
void time_offset_mute_santity(float *tomute, int ntomute);

typedef enum {
  POLY6THCUT = 8,
  TANER4THCUT = 6,
  TANER2TH = 4,
  DSR = 2,
  OTHERS = 2
} TRAVELTIMEMETHOD;
typedef enum { AMPLITUDE = 1, AMPLITUDE_PHASE = 2 } CORRECTION;

typedef struct {
  int sx;
  int sy;
} coor_t;

#ifdef __cplusplus
extern "C" {
#endif

/* Coordinate multiplier of an SU scalco (src/psdmpkg.cc:1013-1028). */
float getscale(short scalco);
/* sx, sy and scalco of nxi velocity traces of `line` (clamped to the last
 * velocity line) from cdp fci on (src/psdmpkg.cc:979-1011). */
void get_vel_coor(const char *velfilepath, int line, coor_t *vel_coor, short *vel_scalel,
                  int fci, int nxi, int fcv, int nxv, int flv, int nyv);
/* Mute depth at an offset: linear between the pairs, the end segments
 * extended outside (src/psdmpkg.cc:1030-1069). */
float time_offset_mute(float *tomute, int ntomute, float offset);

#ifdef __cplusplus
}
#endif

#endif /* QPSDM_PSDMPKG_H_ */
