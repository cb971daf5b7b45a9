// psdmpkg.cpp -- the q-psdm driver's utility API (include/qpsdm_psdmpkg.h),
// written anew with the reference's names, signatures and results
// (src/psdmpkg.cc); each function cites the reference lines it matches.
#include "qpsdm_psdmpkg.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

int xargc;
char **xargv;
int inited;

namespace {

[[noreturn]] void alloc_fail(const char *what, size_t a, size_t b) {
  std::fprintf(stderr, "%s error when call %s(%zu,%zu)\n", what, what, a, b);
  std::exit(0);
}

template <typename T>
T *block(size_t n, const char *what, size_t a, size_t b) {
  T *p = static_cast<T *>(std::malloc(sizeof(T) * (n ? n : 1)));
  if (!p) alloc_fail(what, a, b);
  return p;
}

// rows of n1 elements over one contiguous block of n1 * n2 (p[0] the block)
template <typename T>
T **rows(size_t n1, size_t n2, const char *what) {
  T **p = block<T *>(n2, what, n1, n2);
  p[0] = block<T>(n1 * n2, what, n1, n2);
  for (size_t i = 1; i < n2; ++i) p[i] = p[0] + i * n1;
  return p;
}

}  // namespace

// ---- arrays (src/psdmpkg.cc:24-107, :864-977) ------------------------------
char *malloc1c(size_t n1) { return block<char>(n1, "malloc1c", n1, 0); }
char **malloc2c(size_t n1, size_t n2) { return rows<char>(n1, n2, "malloc2c"); }
int *malloc1i(size_t n1) { return block<int>(n1, "malloc1i", n1, 0); }
int **malloc2i(size_t n1, size_t n2) { return rows<int>(n1, n2, "malloc2i"); }
int ***malloc3i(size_t n1, size_t n2, size_t n3) {
  int ***p = block<int **>(n3, "malloc3i", n1, n2);
  p[0] = rows<int>(n1, n2 * n3, "malloc3i");
  for (size_t i = 1; i < n3; ++i) p[i] = p[0] + i * n2;
  return p;
}
float *malloc1f(size_t n1) { return block<float>(n1, "malloc1f", n1, 0); }
float **malloc2f(size_t n1, size_t n2) { return rows<float>(n1, n2, "malloc2f"); }
float ***malloc3f(size_t n1, size_t n2, size_t n3) {
  float ***p = block<float **>(n3, "malloc3f", n1, n2);
  p[0] = rows<float>(n1, n2 * n3, "malloc3f");
  for (size_t i = 1; i < n3; ++i) p[i] = p[0] + i * n2;
  return p;
}
float ****malloc4f(size_t n1, size_t n2, size_t n3, size_t n4) {
  float ****p = block<float ***>(n4, "malloc4f", n1, n2);
  p[0] = malloc3f(n1, n2, n3 * n4);
  for (size_t i = 1; i < n4; ++i) p[i] = p[0] + i * n3;
  return p;
}
double *malloc1d(size_t n1) { return block<double>(n1, "malloc1d", n1, 0); }
double **malloc2d(size_t n1, size_t n2) { return rows<double>(n1, n2, "malloc2d"); }

// a null row pointer stops the freeing at that level, as the reference's
void free1c(char *p) { std::free(p); }
void free1i(int *p) { std::free(p); }
void free1f(float *p) { std::free(p); }
void free1d(double *p) { std::free(p); }
template <typename T>
static void free_rows(T **p) {
  if (!p) return;
  std::free(p[0]);
  std::free(p);
}
void free2c(char **p) { free_rows(p); }
void free2i(int **p) { free_rows(p); }
void free2f(float **p) { free_rows(p); }
void free2d(double **p) { free_rows(p); }
void free3i(int ***p) {
  if (!p) return;
  free_rows(p[0]);
  std::free(p);
}
void free3f(float ***p) {
  if (!p) return;
  free_rows(p[0]);
  std::free(p);
}
void free4f(float ****p) {
  if (!p) return;
  free3f(p[0]);
  std::free(p);
}

// ---- "a,b-c,d:s:e" (src/psdmpkg.cc:108-204) ---------------------------------
// The items between the markers ',', '-' and ':' are integers (a leading
// integer each, as sscanf "%d" reads it); ',' starts a new item, '-' a range
// from the previous item, ':' a stride, the next ':' its end.
int *parseint(const char *str, int *n) {
  std::vector<char> mark;
  std::vector<int> val(1, 0);
  std::sscanf(str, "%d", &val[0]);
  for (const char *c = str; *c; ++c)
    if (*c == ',' || *c == '-' || *c == ':') {
      mark.push_back(*c);
      int v = 0;
      std::sscanf(c + 1, "%d", &v);
      val.push_back(v);
    }
  std::vector<int> out(1, val[0]);
  for (size_t i = 0; i < mark.size(); ++i) {
    if (mark[i] == ',') {
      out.push_back(val[i + 1]);
    } else if (mark[i] == '-') {
      for (int v = val[i] + 1; v <= val[i + 1]; ++v) out.push_back(v);
    } else if (i + 1 < mark.size()) {  // start ':' stride ':' end
      out.pop_back();
      const int a = val[i], s = val[i + 1], e = val[i + 2];
      if (s > 0)
        for (int v = a; v <= e; v += s) out.push_back(v);
      else if (s < 0)
        for (int v = a; v >= e; v += s) out.push_back(v);
      ++i;
    }
  }
  *n = (int)out.size();
  int *p = static_cast<int *>(std::malloc(sizeof(int) * (out.empty() ? 1 : out.size())));
  std::memcpy(p, out.data(), sizeof(int) * out.size());
  return p;
}

// ---- command line (src/psdmpkg.cc:7-22, :233-336) ---------------------------
void initargs_inner(int argc, char *argv[], const char *sdoc[]) {
  (void)sdoc;
  size_t width = 128 * 1024;
  for (int i = 0; i < argc; ++i) width = std::max(width, std::strlen(argv[i]) + 1);
  xargc = argc;
  xargv = malloc2c(width, (size_t)argc + 1);
  for (int i = 0; i < argc; ++i) std::strcpy(xargv[i], argv[i]);
  inited = 1;
}

static const char *cmdline_value(const char *key) {
  if (!inited) {
    std::fprintf(stderr, "argument is not initialized \n");
    std::exit(0);
  }
  const size_t k = std::strlen(key);
  for (int i = 0; i < xargc; ++i)
    if (std::strncmp(key, xargv[i], k) == 0 && xargv[i][k] == '=') return xargv[i] + k + 1;
  return nullptr;
}
int getparint(const char *key, int *val) {
  const char *v = cmdline_value(key);
  if (!v) return 0;
  *val = (int)std::strtol(v, nullptr, 10);
  return 1;
}
int getparfloat(const char *key, float *val) {
  const char *v = cmdline_value(key);
  if (!v) return 0;
  *val = (float)std::strtod(v, nullptr);
  return 1;
}
int getpardouble(const char *key, double *val) {
  const char *v = cmdline_value(key);
  if (!v) return 0;
  *val = std::strtod(v, nullptr);
  return 1;
}
int getparstr(const char *key, char **val) {
  const char *v = cmdline_value(key);
  if (!v) return 0;
  *val = const_cast<char *>(v);
  return 1;
}
int getparstr(const char *key, const char **val) {
  const char *v = cmdline_value(key);
  if (!v) return 0;
  *val = v;
  return 1;
}

// ---- trace window (src/psdmpkg.cc:208-231) ----------------------------------
int fetch_and_taper(const float *data, int ns, int it1, int it2, float *data1) {
  for (int it = it1; it <= it2; ++it) data1[it - it1] = (it < 0 || it >= ns) ? 0.0f : data[it];
  const int n = it2 - it1 + 1;
  for (int it = 0; it < 200 && it < n; ++it) {
    // the reference's factor: the cosine of the double angle in float
    const float c = (float)(0.5 - 0.5 * cosf((float)(M_PI * it / 200.0)));
    data1[it] *= c;
    data1[n - 1 - it] *= c;
  }
  return 1;
}

// ---- files and strings (src/psdmpkg.cc:206, :601-631) -----------------------
int fexist(const char *path) { return access(path, R_OK | W_OK) == 0; }

size_t fsize(const char *path) {
  struct stat st;
  return stat(path, &st) == 0 ? (size_t)st.st_size : 0;
}

char *strrev1(char *p) {
  if (p) std::reverse(p, p + std::strlen(p));
  return p;
}

char *strrtrim(char *src, int c) {
  if (!src) return src;
  for (size_t i = std::strlen(src); i > 0 && src[i - 1] == c; --i) src[i - 1] = 0;
  return src;
}

// ---- project path (src/psdmpkg.cc:633-684) ----------------------------------
// path = <projpath>/<iproc>/<task>: task the text after the last '/', iproc
// the number between the last two, projpath everything before them and
// projname the last component of projpath.
void parsepath(char *path, char *projpath, char *projname, int *iproc, char *task) {
  const std::string s(path);
  const size_t len = s.size();
  size_t a = s.rfind('/');
  const size_t t0 = a == std::string::npos ? 0 : a + 1;
  std::strcpy(task, s.substr(t0).c_str());
  // the component before the task (stops at the next '/' or the start)
  long i = (long)t0 - 2;
  long b = i;
  while (b >= 0 && s[b] != '/') --b;
  const std::string proc = i >= 0 ? s.substr(b + 1, i - b) : std::string();
  std::strcpy(projpath, s.c_str());
  if (b >= 0) projpath[b] = 0;
  std::sscanf(proc.c_str(), "%d", iproc);
  long c = b - 1;
  long e = c;
  while (e >= 0 && s[e] != '/') --e;
  std::strcpy(projname, c >= 0 ? s.substr(e + 1, c - e).c_str() : "");
  (void)len;
}

// ---- par.dat records (src/psdmpkg.cc:338-574) -------------------------------
namespace {

// The records of a par.dat file: physical lines joined while one ends in a
// backslash (the backslash and the newline removed), leading blanks removed,
// whole-line comments dropped, the text cut at the first '#', trailing blanks
// removed, empty records dropped.
std::vector<std::string> par_records(FILE *fp) {
  std::vector<std::string> recs;
  std::string cur, line;
  char buf[1024];
  auto finish = [&](std::string r) {
    size_t b = 0;
    while (b < r.size() && std::isspace((unsigned char)r[b])) ++b;
    r.erase(0, b);
    if (r.empty() || r[0] == '#') return;
    const size_t h = r.find('#');
    if (h != std::string::npos) r.erase(h);
    while (!r.empty() && std::isspace((unsigned char)r.back())) r.pop_back();
    if (!r.empty()) recs.push_back(r);
  };
  while (std::fgets(buf, sizeof buf, fp)) {
    line += buf;
    if (line.back() != '\n') continue;  // a physical line longer than the buffer
    cur += line;
    line.clear();
    if (cur.size() >= 2 && cur[cur.size() - 2] == '\\') {  // continued
      cur.resize(cur.size() - 2);
      continue;
    }
    cur.pop_back();  // the newline
    finish(cur);
    cur.clear();
  }
  // a last line without a newline is not a record, as the reference reads it
  return recs;
}

}  // namespace

int readparfile(const char *filename, const char *fmt, ...) {
  // patterns "key=%c" separated by commas; every one needs its '=' and '%'
  std::vector<std::string> pats;
  {
    const std::string f(fmt);
    size_t a = 0;
    for (;;) {
      const size_t c = f.find(',', a);
      pats.push_back(f.substr(a, c == std::string::npos ? std::string::npos : c - a));
      if (c == std::string::npos) break;
      a = c + 1;
    }
    size_t neq = 0, npc = 0;
    for (char ch : f) neq += ch == '=', npc += ch == '%';
    if (pats.size() != neq || neq != npc) {
      std::fprintf(stderr, "Error: In FUNCTION: %s fmt[%s] [, = %%] do not Match\n",
                   __func__, fmt);
      std::exit(0);
    }
  }
  FILE *fp = std::fopen(filename, "r");
  if (!fp) {
    std::fprintf(stderr, "Error: Parameter File [%s] Open Error\n", filename);
    std::exit(0);
  }
  const std::vector<std::string> recs = par_records(fp);
  std::fclose(fp);
  va_list ap;
  va_start(ap, fmt);
  int nret = 0, result = 0;
  const int npat = (int)pats.size();
  for (const std::string &pat : pats) {
    int matches = 0;
    const char conv = pat.empty() ? 0 : pat.back();
    for (const std::string &rec : recs) {
      bool hit = false;
      int iv = 0;
      float fv = 0.0f;
      std::vector<char> sv(rec.size() + 1);
      switch (conv) {
        case 'd':
          hit = std::sscanf(rec.c_str(), pat.c_str(), &iv) == 1;
          break;
        case 'f':
        case 'g':
          hit = std::sscanf(rec.c_str(), pat.c_str(), &fv) == 1;
          break;
        case 's':
          hit = std::sscanf(rec.c_str(), pat.c_str(), sv.data()) == 1;
          break;
        case 'S':  // the literal part ("key=") starts the record
          hit = rec.compare(0, pat.size() - 2, pat, 0, pat.size() - 2) == 0;
          break;
        default:
          break;
      }
      if (!hit) continue;
      ++matches;
      if (nret >= npat) {  // more matches than outputs: the reference stops here
        va_end(ap);
        return -1;
      }
      switch (conv) {
        case 'd':
          *va_arg(ap, int *) = iv;
          break;
        case 'f':
        case 'g':
          *va_arg(ap, float *) = fv;
          break;
        case 's': {  // at most 1023 characters, as the reference copies
          char *out = va_arg(ap, char *);
          const size_t n = std::min<size_t>(std::strlen(sv.data()), 1023);
          std::memcpy(out, sv.data(), n);
          out[n] = 0;
          break;
        }
        default: {  // 'S': the rest of the record, malloc'd
          const std::string rest = rec.substr(pat.size() - 2);
          char *p = static_cast<char *>(std::malloc(rest.size() + 1));
          std::memcpy(p, rest.c_str(), rest.size() + 1);
          *va_arg(ap, char **) = p;
        }
      }
      ++nret;
    }
    if (matches != 1) result = -1;
  }
  va_end(ap);
  return result < 0 ? -1 : nret;
}

// ---- tuples (src/psdmpkg.cc:686-862) ----------------------------------------
// A number is a run of digits, '.', 'e', 'E' (and here a sign); blanks,
// tabs, ',' and ';' separate numbers.
float *parsetuple(const char *str, int *ntuple, int *nelem) {
  const std::string s(str);
  const long nl = std::count(s.begin(), s.end(), '('), nr = std::count(s.begin(), s.end(), ')');
  *ntuple = 0;
  *nelem = 0;
  if (nl != nr || nl == 0) {
    std::fprintf(stderr, "Warn: String [%s]'s brackets do not match,or has no element\n", str);
    return nullptr;
  }
  auto numch = [](char c) {
    return (c >= '0' && c <= '9') || c == '.' || c == 'e' || c == 'E' || c == '-' || c == '+';
  };
  std::vector<std::vector<float>> tup;
  size_t l = 0, r = 0;
  for (;;) {  // the k-th '(' pairs with the k-th ')', as the reference pairs them
    l = s.find('(', l);
    r = s.find(')', r);
    if (l == std::string::npos || r == std::string::npos) break;
    std::vector<float> v;
    for (size_t i = l + 1; i < r;) {
      if (numch(s[i])) {
        size_t j = i;
        while (j < r && numch(s[j])) ++j;
        float x;
        if (std::sscanf(s.substr(i, j - i).c_str(), "%f", &x) != 1) {
          std::fprintf(stderr, "Error: Elements Parse Error\n");
          return nullptr;
        }
        v.push_back(x);
        i = j;
      } else {
        ++i;
      }
    }
    tup.push_back(v);
    ++l;
    ++r;
  }
  for (const auto &v : tup)
    if (v.size() != tup[0].size()) {
      std::fprintf(stderr, "Error: String [%s]'s Elements Count do not match\n", str);
      return nullptr;
    }
  const size_t ne = tup[0].size();
  float *p = static_cast<float *>(std::malloc(sizeof(float) * (tup.size() * ne + 1)));
  for (size_t k = 0; k < tup.size(); ++k)
    std::memcpy(p + k * ne, tup[k].data(), sizeof(float) * ne);
  *ntuple = (int)tup.size();
  *nelem = (int)ne;
  return p;
}

// ---- mute (src/psdmpkg.cc:576-599, :1030-1069) ------------------------------
void time_offset_mute_santity(float *m, int n) {
  // mirror a decreasing pair about the previous one, then force strictly
  // increasing pairs (depth + 0.01, offset + 10), in double as the reference
  for (int i = 0; i + 1 < n; ++i) {
    if (m[2 * i] > m[2 * i + 2]) m[2 * i + 2] = (float)(2.0 * m[2 * i] - m[2 * i + 2]);
    if (m[2 * i + 1] > m[2 * i + 3]) m[2 * i + 3] = (float)(2.0 * m[2 * i + 1] - m[2 * i + 3]);
  }
  for (int i = 0; i + 1 < n; ++i) {
    if (m[2 * i] >= m[2 * i + 2]) m[2 * i + 2] = (float)(m[2 * i] + 0.01);
    if (m[2 * i + 1] >= m[2 * i + 3]) m[2 * i + 3] = (float)(m[2 * i + 1] + 10.0);
  }
}

extern "C" float time_offset_mute(float *m, int n, float o) {
  if (n < 2) return m[0];
  int a = -1;
  if (o < m[1])
    a = 0;
  else if (o >= m[2 * (n - 1) + 1])
    a = n - 2;
  else
    for (int i = 0; i + 1 < n; ++i)
      if (m[2 * i + 1] <= o && o < m[2 * i + 3]) a = i;  // the last pair that holds o
  if (a < 0) return 0.0f;  // offsets not increasing: no pair holds o
  const float o1 = m[2 * a + 1], o2 = m[2 * a + 3], t1 = m[2 * a], t2 = m[2 * a + 2];
  return t1 + (t2 - t1) / (o2 - o1) * (o - o1);
}

// ---- coordinates (src/psdmpkg.cc:979-1028) ----------------------------------
extern "C" float getscale(short scalco) {
  if (scalco == 0) return 1.0f;
  return scalco > 0 ? (float)scalco : (float)(-1.0 / scalco);
}

extern "C" void get_vel_coor(const char *velfilepath, int line, coor_t *vel_coor,
                             short *vel_scalel, int fci, int nxi, int fcv, int nxv, int flv,
                             int nyv) {
  FILE *fp = std::fopen(velfilepath, "rb");
  if (!fp) {
    std::fprintf(stderr, "Velocity File open Error\n");
    std::exit(1);
  }
  segy *tr = static_cast<segy *>(std::malloc(sizeof(segy)));
  fgettr(fp, tr);
  *vel_scalel = tr->scalco;
  if (line >= flv + nyv) line = flv + nyv - 1;
  std::fseek(fp, (long)(sizeof(float) * tr->ns + 240L) * ((line - flv) * nxv + fci - fcv),
             SEEK_SET);
  for (int i = 0; i < nxi; ++i) {
    fgettr(fp, tr);
    vel_coor[i].sx = tr->sx;
    vel_coor[i].sy = tr->sy;
  }
  std::free(tr);
  std::fclose(fp);
}
