// q-psdm -- the command-line driver of the B200 imaging engine.
//
// A drop-in for the reference program's driver (src/q-psdm.cu:383-1160 main,
// :1161-1860 qpsdm, :1862-1926 producer): the same command-line keys and
// par.dat keys with the same defaults, the same project layout
//   <path> = <projpath>/<iproc>/<task>
//   <projpath>/data<idata>/nofffile.rcd            "nofffile=N"
//   <projpath>/data<idata>/off<k>/ell_off<k>        "offmin,offmax"
//   <projpath>/data<idata>/off<k>/line<l>           input SU (big-endian)
//   <ttpath>/Lxxx.{tidx,qidx}, <ttpath>/L<line>.{ttt,qqq}
//   <projpath>/<idata>/<task>/result/<node>_<idata>.off<k>.L<line>.su   output
// and the same checkpoint markers (<offspath>/break_point.txt holding the
// last finished line, an empty <infopath>/<node>_<line> per line, an empty
// <infopath of data 0>/<node> at the end).  The imaging itself goes through
// the engine's C ABI (include/qpsdm_engine.h); a reader thread fills pinned
// host buffers with raw SU records while the engine images the previous one.
//
// Keys this driver adds (the reference has no counterpart):
//   engine=compat|physics   compat (default) reproduces the reference's stub
//                           kernel; physics images with the t / t* tables
//   form=plain|batched      physics form (default batched)
//   panels=fp32|bf16|fp16   physics panel type (default fp16 batched, fp32 plain)
//   nbins=16 dtstar=0.002   t* bins of the compensated panels
//   aperx, apery            half aperture in cdps / lines for every azimuth
//                           (the reference allocates but never fills its
//                           aperture tables, src/q-psdm.cu:1542-1545;
//                           default: the whole image)
//   dzii                    table depth-node spacing (default 48 m as the
//                           reference derives it, src/q-psdm.cu:880-882)
//   max_batch               traces per submit (default 16384)
//   brick=N                 image N consecutive lines of the line list in one
//                           pass over the data (default 1, as the reference;
//                           each data line still feeds only the image lines
//                           within +-extxline of it)
//   resume=1                skip the lines up to <offspath>/break_point.txt
//   check=1                 resolve and print the parameters, image nothing
//   check=2                 also load every line's tables and list the data files
//                           (whole traces, trailing partial bytes), image nothing
// Errors print a message and exit 1, as the reference does; the library
// itself never exits.
#include <cuda_runtime.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <condition_variable>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "qpsdm_engine.h"
#include "qpsdm_psdmpkg.h"

namespace {

[[noreturn]] void die(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::fprintf(stderr, "Error: ");
  std::vfprintf(stderr, fmt, ap);
  std::fprintf(stderr, "\n");
  va_end(ap);
  std::exit(1);
}

void logf(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vfprintf(stderr, fmt, ap);
  va_end(ap);
}

bool exists(const std::string &p) { return access(p.c_str(), F_OK) == 0; }

// ---------------------------------------------------------------------------
// command line and par.dat, through libqpsdm_pkg (include/qpsdm_psdmpkg.h)
// ---------------------------------------------------------------------------
// A key is taken from the command line first (getpar*), else from par.dat,
// where exactly one record must match the typed pattern "key=%d" / "key=%f"
// / "key=%s" (src/q-psdm.cu:425-871: getparX(k) || readparfile(...) == 1).
struct Keys {
  std::string parfile;
  bool str(const char *k, std::string &out) const {
    char *v = nullptr;
    if (getparstring(k, &v)) {
      out = v;
      return true;
    }
    char buf[1024];
    if (readparfile(parfile.c_str(), (std::string(k) + "=%s").c_str(), buf) != 1) return false;
    out = buf;
    return true;
  }
  bool num(const char *k, int &out) const {
    return getparint(k, &out) || readparfile(parfile.c_str(), (std::string(k) + "=%d").c_str(), &out) == 1;
  }
  bool num(const char *k, float &out) const {
    return getparfloat(k, &out) || readparfile(parfile.c_str(), (std::string(k) + "=%f").c_str(), &out) == 1;
  }
  std::string str_or(const char *k, const std::string &def) const {
    std::string v;
    return str(k, v) ? v : def;
  }
  std::string str_req(const char *k) const {
    std::string v;
    if (!str(k, v)) die("%s must be specified", k);
    return v;
  }
  int int_or(const char *k, int def) const {
    int v = def;
    return num(k, v) ? v : def;
  }
  int int_req(const char *k) const {
    int v = 0;
    if (!num(k, v)) die("%s must be specified", k);
    return v;
  }
  float flt_or(const char *k, float def) const {
    float v = def;
    return num(k, v) ? v : def;
  }
  float flt_req(const char *k) const {
    float v = 0.0f;
    if (!num(k, v)) die("%s must be specified", k);
    return v;
  }
};

// "1,5-8,10:2:16" -> 1 5 6 7 8 10 12 14 16 (parseline)
std::vector<int> parse_list(const std::string &s) {
  int n = 0;
  int *p = parseline(s.c_str(), &n);
  std::vector<int> out(p, p + std::max(n, 0));
  std::free(p);
  return out;
}

// "(d1,o1),(d2,o2)..." -> the (depth, offset) pairs made increasing
// (parsetuple + time_offset_mute_santity, src/q-psdm.cu:1014-1025)
std::vector<float> mute_pairs(const std::string &s) {
  int nt = 0, ne = 0;
  float *p = parsetuple(s.c_str(), &nt, &ne);
  if (!p || ne != 2 || nt < 1) die("mute [%s] is not a list of (depth,offset) pairs", s.c_str());
  std::vector<float> m(p, p + 2 * nt);
  std::free(p);
  time_offset_mute_santity(m.data(), nt);
  return m;
}
float mute_depth(std::vector<float> &m, float o) {
  return time_offset_mute(m.data(), (int)m.size() / 2, o);
}

// <projpath>/<iproc>/<task>, trailing '/' removed first (strrtrim +
// parsepath, src/q-psdm.cu:396-420)
struct ProjPath {
  std::string projpath, projname, task;
  int iproc = 0;
};
ProjPath parse_path(std::string &path) {
  std::vector<char> buf(path.begin(), path.end());
  buf.push_back(0);
  strrtrim(buf.data(), '/');
  path = buf.data();
  const size_t n = buf.size() + 1;
  std::vector<char> pp(n, 0), pn(n, 0), task(n, 0);
  ProjPath r;
  parsepath(buf.data(), pp.data(), pn.data(), &r.iproc, task.data());
  r.projpath = pp.data();
  r.projname = pn.data();
  r.task = task.data();
  return r;
}

// ---------------------------------------------------------------------------
// SU records (big-endian on disk, SEG-Y trace header offsets)
// ---------------------------------------------------------------------------
constexpr int kHdr = 240;
enum { oTracl = 0, oFldr = 8, oCdp = 20, oTrid = 28, oNvs = 30, oOffset = 36, oScalco = 70,
       oSx = 72, oSy = 76, oGx = 80, oGy = 84, oCounit = 88, oNs = 114, oDt = 116 };

int32_t be_i32(const uint8_t *p) {
  return (int32_t)((uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]);
}
int16_t be_i16(const uint8_t *p) { return (int16_t)((uint16_t)p[0] << 8 | p[1]); }
void put_i32(uint8_t *p, int32_t v) {
  const uint32_t u = (uint32_t)v;
  p[0] = u >> 24;
  p[1] = u >> 16;
  p[2] = u >> 8;
  p[3] = u;
}
void put_i16(uint8_t *p, int16_t v) {
  const uint16_t u = (uint16_t)v;
  p[0] = u >> 8;
  p[1] = u;
}

struct TraceHdr {
  uint8_t h[kHdr];
};
// header of trace k of an SU file whose traces have ns samples
bool read_header(FILE *fp, long k, int ns, TraceHdr &t) {
  if (std::fseek(fp, k * (kHdr + 4L * ns), SEEK_SET) != 0) return false;
  return std::fread(t.h, 1, kHdr, fp) == (size_t)kHdr;
}
// ---------------------------------------------------------------------------
// tables: Lxxx.{tidx,qidx} + L<line>.{ttt,qqq}, inter-line lerp
// (get_ttt_all, src/q-psdm.cu:2382-2622)
// ---------------------------------------------------------------------------
struct Tables {
  int cdp1 = 0, cdp2 = 0, nzg = 0, nxg = 0, nzi1 = 0, nxi1 = 0;
  std::vector<qpsdm_ttt_desc> desc;
  std::vector<float> data;     // values of the bracketing line lo
  std::vector<float> data_hi;  // values of line hi (empty when the line has its own file)
  int lo = 0, hi = 0;
  float *d = nullptr;          // the line's values on the device (tables_on_device)
  Tables() = default;
  Tables(const Tables &) = delete;
  Tables &operator=(const Tables &) = delete;
  ~Tables() {
    if (d) cudaFree(d);
  }
};
bool load_tables(const std::string &ttpath, bool q, int line, int line1, int line2, Tables &t) {
  const std::string idx = ttpath + (q ? "/Lxxx.qidx" : "/Lxxx.tidx");
  const char *suff = q ? "qqq" : "ttt";
  FILE *fp = std::fopen(idx.c_str(), "rb");
  if (!fp) return false;
  int32_t h[2];
  float dxdz[2];
  int32_t g[4];
  bool ok = std::fread(h, 4, 2, fp) == 2 && std::fread(dxdz, 4, 2, fp) == 2 &&
            std::fread(g, 4, 4, fp) == 4;
  if (ok) {
    t.cdp1 = h[0];
    t.cdp2 = h[1];
    t.nzg = g[0];
    t.nxg = g[1];
    t.nzi1 = g[2];
    t.nxi1 = g[3];
    // a header whose grid does not fit the file is an index size error
    // before anything is allocated for it
    struct stat st;
    const long long ncell = (long long)t.nxg * t.nzg;
    ok = t.nxg > 0 && t.nzg > 0 && t.nzi1 > 0 && t.nxi1 > 0 &&
         fstat(fileno(fp), &st) == 0 &&
         (long long)st.st_size >= 32 + ncell * (long long)sizeof(qpsdm_ttt_desc);
    if (ok) {
      t.desc.resize((size_t)ncell);
      ok = std::fread(t.desc.data(), sizeof(qpsdm_ttt_desc), t.desc.size(), fp) == t.desc.size();
    }
  }
  std::fclose(fp);
  if (!ok) die("travel time table or qfield index size error %s", idx.c_str());
  auto path_of = [&](int l) { return ttpath + "/L" + std::to_string(l) + "." + suff; };
  int lo = -1, hi = -1;
  for (int l = line; l >= line1; --l)
    if (exists(path_of(l))) {
      lo = l;
      break;
    }
  for (int l = line; l <= line2; ++l)
    if (exists(path_of(l))) {
      hi = l;
      break;
    }
  if (lo < 0 || hi < 0) die("no %s table brackets line %d in %s", suff, line, ttpath.c_str());
  auto read_all = [&](int l, std::vector<float> &v) {
    FILE *f = std::fopen(path_of(l).c_str(), "rb");
    if (!f) die("cannot open %s", path_of(l).c_str());
    std::fseek(f, 0, SEEK_END);
    const long bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize((size_t)bytes / 4);
    if (std::fread(v.data(), 4, v.size(), f) != v.size()) die("read %s", path_of(l).c_str());
    std::fclose(f);
  };
  read_all(lo, t.data);
  t.lo = lo;
  t.hi = hi;
  t.data_hi.clear();
  if (hi != lo) {
    read_all(hi, t.data_hi);
    if (t.data_hi.size() != t.data.size()) die("table sizes of lines %d and %d differ", lo, hi);
  }
  return true;
}

// The line's table values on the current device: line lo's values, or the
// interpolation between lines lo and hi with get_ttt_all's float arithmetic
// (src/q-psdm.cu:2584-2596), computed on the GPU by qpsdm_tables_lerp
// instead of a host loop over the tens of millions of values of a line.
// The host copies are released; the engine copies the device values at
// qpsdm_set_lines.
float *tables_on_device(Tables &t, int line) {
  const size_t n = t.data.size(), bytes = n * sizeof(float);
  auto ck = [&](cudaError_t c, const char *what) {
    if (c != cudaSuccess) die("tables of line %d: %s: %s", line, what, cudaGetErrorString(c));
  };
  ck(cudaMalloc(&t.d, bytes ? bytes : sizeof(float)), "cudaMalloc");
  if (t.data_hi.empty()) {
    ck(cudaMemcpy(t.d, t.data.data(), bytes, cudaMemcpyHostToDevice), "upload");
  } else {
    float *d_lo = nullptr, *d_hi = nullptr;
    ck(cudaMalloc(&d_lo, bytes), "cudaMalloc");
    ck(cudaMalloc(&d_hi, bytes), "cudaMalloc");
    ck(cudaMemcpy(d_lo, t.data.data(), bytes, cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(d_hi, t.data_hi.data(), bytes, cudaMemcpyHostToDevice), "upload");
    if (qpsdm_tables_lerp(d_lo, d_hi, (int64_t)n, line, t.lo, t.hi, t.d, nullptr) != QPSDM_OK)
      die("tables of line %d: qpsdm_tables_lerp failed", line);
    ck(cudaDeviceSynchronize(), "interpolation");
    cudaFree(d_lo);
    cudaFree(d_hi);
  }
  std::vector<float>().swap(t.data);
  std::vector<float>().swap(t.data_hi);
  return t.d;
}

// ---------------------------------------------------------------------------
// producer: a reader thread filling pinned buffers with raw SU records
// ---------------------------------------------------------------------------
class Producer {
 public:
  Producer(size_t rec_bytes, int max_batch, int nbuf) : rec_bytes_(rec_bytes), max_(max_batch) {
    for (int i = 0; i < nbuf; ++i) {
      void *p = nullptr;
      if (cudaMallocHost(&p, rec_bytes * max_batch) != cudaSuccess)
        die("pinned host buffer of %zu bytes", rec_bytes * max_batch);
      bufs_.push_back((uint8_t *)p);
      free_.push_back(i);
    }
  }
  ~Producer() {
    if (th_.joinable()) th_.join();
    for (auto *p : bufs_) cudaFreeHost(p);
  }
  // start reading the files (path, data line) in order
  void start(std::vector<std::pair<std::string, int>> files) {
    done_ = false;
    th_ = std::thread([this, files] { run(files); });
  }
  // next filled buffer (index, traces, data line); false when all are read
  bool next(int &buf, int &ntr, int &line) {
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return !full_.empty() || done_; });
    if (full_.empty()) return false;
    buf = full_.front().buf;
    ntr = full_.front().n;
    line = full_.front().line;
    full_.pop_front();
    return true;
  }
  void release(int buf) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      free_.push_back(buf);
    }
    cv_.notify_all();
  }
  void join() {
    if (th_.joinable()) th_.join();
  }
  const uint8_t *data(int buf) const { return bufs_[buf]; }
  long traces_read = 0;

 private:
  void run(std::vector<std::pair<std::string, int>> files) {
    for (const auto &fl : files) {
      const std::string &f = fl.first;
      FILE *fp = std::fopen(f.c_str(), "rb");
      if (!fp) continue;  // a missing data line contributes nothing
      struct stat st;
      fstat(fileno(fp), &st);
      // whole records only, as the reference's producer (src/q-psdm.cu:1909)
      long left = (long)(st.st_size / (long)rec_bytes_);
      if (st.st_size % (long)rec_bytes_)
        logf("Warn: %s ends in a partial trace (%ld bytes), ignored\n", f.c_str(),
             (long)(st.st_size % (long)rec_bytes_));
      while (left > 0) {
        int b;
        {
          std::unique_lock<std::mutex> lk(mu_);
          cv_.wait(lk, [&] { return !free_.empty(); });
          b = free_.front();
          free_.pop_front();
        }
        const int n = (int)std::min<long>(left, max_);
        const size_t got = std::fread(bufs_[b], rec_bytes_, n, fp);
        if ((int)got != n) die("Read %s fail: %s", f.c_str(), std::strerror(errno));
        left -= n;
        traces_read += n;
        {
          std::lock_guard<std::mutex> lk(mu_);
          full_.push_back({b, n, fl.second});
        }
        cv_.notify_all();
      }
      std::fclose(fp);
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      done_ = true;
    }
    cv_.notify_all();
  }
  size_t rec_bytes_;
  int max_;
  std::vector<uint8_t *> bufs_;
  std::deque<int> free_;
  struct Filled {
    int buf, n, line;
  };
  std::deque<Filled> full_;
  bool done_ = true;
  std::mutex mu_;
  std::condition_variable cv_;
  std::thread th_;
};

void touch(const std::string &p, const std::string &content) {
  FILE *fp = std::fopen(p.c_str(), "w");
  if (fp) {
    std::fputs(content.c_str(), fp);
    std::fclose(fp);
  }
}

void check_engine(int rc, qpsdm_engine *e, const char *what) {
  if (rc != QPSDM_OK) die("%s failed (%d): %s", what, rc, e ? qpsdm_last_error(e) : "");
}

}  // namespace

int main(int argc, char **argv) {
  initargs_inner(argc, argv, nullptr);
  auto cmd = [](const char *k) {
    char *v = nullptr;
    if (!getparstring(k, &v)) die("%s must be specified", k);
    return std::string(v);
  };
  std::string path = cmd("path");
  const std::string parfilepath = cmd("parfilepath"), nodename = cmd("nodename"),
                    ttpath = cmd("ttpath");
  FILE *pf = std::fopen(parfilepath.c_str(), "r");
  if (!pf) die("Parameter File [%s] Open Error", parfilepath.c_str());
  std::fclose(pf);
  Keys K{parfilepath};
  const ProjPath pp = parse_path(path);

  // ---- keys (src/q-psdm.cu:433-714) ----
  std::string offspath = K.str_or("offspath", pp.projpath + "/data" + std::to_string(pp.iproc));
  const std::string velfilepath = K.str_or("velfilepath", pp.projpath + "/vel/vel_loadin");
  std::string infopath = K.str_or("infopath", path);
  const float fc = K.flt_or("fc", 40.0f), contract = K.flt_or("contract", 3.0f);
  const float taperzone = K.flt_or("taperzone", 8.0f), threshold = K.flt_or("threshold", 600.0f);
  const float f1 = K.flt_or("f1", 1.0f);
  float f3 = K.flt_or("f3", 130.0f), f4 = K.flt_or("f4", 140.0f);
  const int ntl = K.int_req("ntl");
  const float dt = K.flt_req("dt");
  const int line1 = K.int_req("line1"), line2 = K.int_req("line2");
  const float zmin = K.flt_req("zmin"), zmax = K.flt_req("zmax"), dzi = K.flt_req("dzi");
  const int cdp1 = K.int_req("cdp1"), cdp2 = K.int_req("cdp2");
  const std::vector<int> lines = parse_list(K.str_req("line"));
  const std::string zmute = K.str_or("mute", "(1,9999),(100,9999)");
  const int xline = K.int_req("extxline");
  const int opcrp = K.int_or("opcrp", 0);
  const std::vector<int> cdps =
      parse_list(K.str_or("cdps", std::to_string(cdp1) + "-" + std::to_string(cdp2)));
  const int nblock = std::max(1, K.int_or("nblock", 1));
  // the reference reads ndata but clamps it to its GPU count, which it sets
  // to 1 (src/q-psdm.cu:786-798): one data directory, data<iproc>'s sibling 0
  const int ndata = std::min(std::max(1, K.int_or("ndata", 1)), 1);
  // Nyquist clamps (src/q-psdm.cu:711-723)
  if (f3 > 0.5f / dt - 10.0f) f3 = 0.5f / dt - 10.0f;
  if (f4 > 0.5f / dt - 5.0f) f4 = 0.5f / dt - 5.0f;
  if (f4 - f3 <= 5.0f) f3 = f4 - 5.0f;
  // this driver's keys
  const std::string engine_mode = K.str_or("engine", "compat");
  const std::string form = K.str_or("form", "batched");
  const std::string panels = K.str_or("panels", form == "plain" ? "fp32" : "fp16");
  const int nbins = K.int_or("nbins", 16);
  const float dtstar = K.flt_or("dtstar", 0.002f);
  const int max_batch = std::max(1, K.int_or("max_batch", 16384));
  const int resume = K.int_or("resume", 0);
  const int brick = std::min(std::max(1, K.int_or("brick", 1)), 64);
  const int check_only = K.int_or("check", 0);
  if (engine_mode != "compat" && engine_mode != "physics") die("engine must be compat or physics");
  if (form != "plain" && form != "batched") die("form must be plain or batched");
  if (panels != "fp32" && panels != "bf16" && panels != "fp16") die("panels must be fp32, bf16 or fp16");

  // GPU from the node name "<name>_<gpu>" (src/q-psdm.cu:725-786)
  int igpu = 0;
  if (std::sscanf(nodename.c_str(), "%*[^_]_%d", &igpu) != 1)
    die("Nodename [%s] Format Error or This Machine has no GPUs", nodename.c_str());
  const std::string node0 = nodename.substr(0, nodename.find('_'));

  // image space (src/q-psdm.cu:826-834)
  const int fci = cdp1, nxi = cdp2 - cdp1 + 1, nyi = (int)lines.size();
  const int nzi = (int)(zmax / dzi + 0.5f) + 1;
  if (nxi <= 0 || nzi <= 0 || nyi <= 0) die("empty image (cdp1..cdp2, zmax, line)");

  // velocity-file geometry: first and last trace (src/q-psdm.cu:836-880)
  if (!exists(velfilepath)) die("On Node [%s], Velocity File [%s] Does Not Exist", nodename.c_str(),
                                velfilepath.c_str());
  FILE *vf = std::fopen(velfilepath.c_str(), "rb");
  TraceHdr v0, v1;
  if (!vf || std::fread(v0.h, 1, kHdr, vf) != (size_t)kHdr) die("velocity file header");
  const int ntv = (uint16_t)be_i16(v0.h + oNs);
  std::fseek(vf, -(long)(kHdr + 4L * ntv), SEEK_END);
  if (std::fread(v1.h, 1, kHdr, vf) != (size_t)kHdr) die("velocity file last header");
  // float arithmetic as src/q-psdm.cu:846-858 (int x float -> float)
  const float scalev = getscale(be_i16(v0.h + oScalco));
  const double fxv = (float)be_i32(v0.h + oGx) * scalev;
  const double fyv = (float)be_i32(v0.h + oGy) * scalev;
  const int fcv = be_i32(v0.h + oCdp), flv = be_i32(v0.h + oFldr);
  const int nxv = be_i32(v1.h + oCdp) - fcv + 1, nyv = be_i32(v1.h + oFldr) - flv + 1;
  if (nxv < 2) die("velocity file has a single cdp");
  const float dxv = (float)(be_i32(v1.h + oGx) - be_i32(v0.h + oGx)) * scalev / (float)(nxv - 1);
  float dyv;
  if (nyv == 1) {
    if (!K.num("dyv", dyv))
      die("since first fldr and last fldr in the velocity file is the same:%d please specify dyv!",
          flv);
  } else {
    dyv = (float)(be_i32(v1.h + oGy) - be_i32(v0.h + oGy)) * scalev / (float)(nyv - 1);
    dyv = K.flt_or("dyv", dyv);
  }
  const float dxi = dxv, dyi = dyv;
  const float dzii = K.flt_or("dzii", 8.0f * std::round(50.0f / 8.0f));
  const int aperx = K.int_or("aperx", nxi), apery = K.int_or("apery", nyv);

  // data-space scale and sanity (src/q-psdm.cu:886-915)
  double scaled = 1.0;
  for (int l = lines[0] - 1000; l < lines[0] + 1000; ++l) {
    const std::string f = offspath + "/off0/line" + std::to_string(l);
    if (!exists(f)) continue;
    FILE *fp = std::fopen(f.c_str(), "rb");
    TraceHdr t;
    if (fp && std::fread(t.h, 1, kHdr, fp) == (size_t)kHdr) {
      scaled = getscale(be_i16(t.h + oScalco));
      if ((uint16_t)be_i16(t.h + oNs) != ntl)
        die("In Data Space (tr.ns=%d)!=(ntl=%d)", (uint16_t)be_i16(t.h + oNs), ntl);
      if ((uint16_t)be_i16(t.h + oDt) != (int)(dt * 1.0E6f))
        die("In Data Space (tr.dt=%d)!=(dt=%g*1.0E6)", (uint16_t)be_i16(t.h + oDt), dt);
    }
    if (fp) std::fclose(fp);
    break;
  }

  // offset groups of each data directory (src/q-psdm.cu:917-972)
  std::vector<std::vector<float>> offmin(ndata), offmax(ndata);
  for (int id = 0; id < ndata; ++id) {
    const std::string op = pp.projpath + "/data" + std::to_string(id);
    const std::string rcd = op + "/nofffile.rcd";
    FILE *fp = std::fopen(rcd.c_str(), "r");
    int n = 0;
    if (!fp || std::fscanf(fp, "nofffile=%d", &n) != 1)
      die("On %s_%d,[%s] Does Not Exist or unreadable", node0.c_str(), id, rcd.c_str());
    std::fclose(fp);
    for (int k = 0; k < n; ++k) {
      const std::string e = op + "/off" + std::to_string(k) + "/ell_off" + std::to_string(k);
      FILE *f = std::fopen(e.c_str(), "r");
      float a, b;
      if (!f || std::fscanf(f, "%f,%f", &a, &b) != 2) die("Read offmin and offmax from %s fail!", e.c_str());
      std::fclose(f);
      offmin[id].push_back(a);
      offmax[id].push_back(b);
    }
  }
  auto mute = mute_pairs(zmute);

  logf("q-psdm: node %s gpu %d  image %d cdps x %d lines x %d depths  dx %g dy %g dz %g\n",
       nodename.c_str(), igpu, nxi, nyi, nzi, dxi, dyi, dzi);
  logf("        velocity grid fxv %.3f fyv %.3f fcv %d flv %d nxv %d nyv %d; data scale %g\n", fxv,
       fyv, fcv, flv, nxv, nyv, scaled);
  logf("        engine %s form %s panels %s nbins %d dtstar %g aperture %d x %d opcrp %d\n",
       engine_mode.c_str(), form.c_str(), panels.c_str(), nbins, dtstar, aperx, apery, opcrp);

  // ---- engine (src/q-psdm.cu:1161-1376) ----
  qpsdm_static_params sp;
  std::memset(&sp, 0, sizeof sp);
  sp.dyi = dyi;
  sp.dxi = dxi;
  sp.nxi = nxi;
  sp.nzi = nzi;
  sp.ntl = ntl;
  sp.scaled = scaled;
  sp.fci = fci;
  sp.dzi = dzi;
  sp.dt = dt;
  sp.fc = fc;
  sp.f1 = f1;
  sp.f3 = f3;
  sp.f4 = f4;
  sp.threshold = threshold;
  sp.contract = contract;
  sp.taperzone = taperzone;
  sp.fxv1 = (float)(fxv - 2000.0);
  sp.exv1 = (float)(fxv + nxv * dxi + 2000.0);
  sp.fyv1 = (float)(fyv - 1000.0);
  sp.eyv1 = (float)(fyv + nyv * dyi + 1000.0);
  sp.dzii = dzii;
  sp.mode = engine_mode == "physics" ? QPSDM_MODE_PHYSICS : QPSDM_MODE_COMPAT;
  sp.panel_dtype = panels == "fp32" ? QPSDM_PANEL_FP32
                   : panels == "bf16" ? QPSDM_PANEL_BF16 : QPSDM_PANEL_FP16;
  sp.nbins = nbins;
  sp.dtstar = dtstar;
  sp.max_batch = max_batch;
  sp.form = form == "plain" ? QPSDM_FORM_PLAIN : QPSDM_FORM_BATCHED;
  if (qpsdm_static_params_init(&sp) != QPSDM_OK) die("bad parameters");
  logf("        nfft %d nffti %d dt1 %g contract %g taperzone %g (rad)\n", sp.nfft, sp.nffti,
       sp.dt1, sp.contract, sp.taperzone);
  if (check_only) {
    std::printf("{\"projpath\":\"%s\",\"projname\":\"%s\",\"iproc\":%d,\"task\":\"%s\","
                "\"offspath\":\"%s\",\"velfilepath\":\"%s\",\"infopath\":\"%s\","
                "\"nxi\":%d,\"nyi\":%d,\"nzi\":%d,\"fci\":%d,\"dxi\":%.9g,\"dyi\":%.9g,"
                "\"fxv\":%.17g,\"fyv\":%.17g,\"fcv\":%d,\"flv\":%d,\"nxv\":%d,\"nyv\":%d,"
                "\"scaled\":%.17g,\"f1\":%.6g,\"f3\":%.6g,\"f4\":%.6g,\"fc\":%.6g,"
                "\"threshold\":%.6g,\"contract_deg\":%.6g,\"taperzone_deg\":%.6g,"
                "\"extxline\":%d,\"opcrp\":%d,\"aperx\":%d,\"apery\":%d,\"dzii\":%.6g,"
                "\"engine\":\"%s\",\"form\":\"%s\",\"panels\":\"%s\",\"nbins\":%d,"
                "\"dtstar\":%.6g,\"max_batch\":%d,\"nblock\":%d,\"gpu\":%d,\"node0\":\"%s\","
                "\"noffs\":%d,\"offmin\":%.6g,\"offmax\":%.6g,\"nfft\":%d,\"nffti\":%d,"
                "\"lines\":[",
                pp.projpath.c_str(), pp.projname.c_str(), pp.iproc, pp.task.c_str(),
                offspath.c_str(), velfilepath.c_str(), infopath.c_str(), nxi, nyi, nzi, fci, dxi,
                dyi, fxv, fyv, fcv, flv, nxv, nyv, scaled, f1, f3, f4, fc, threshold, contract,
                taperzone, xline, opcrp, aperx, apery, dzii, engine_mode.c_str(), form.c_str(),
                panels.c_str(), nbins, dtstar, max_batch, nblock, igpu, node0.c_str(),
                (int)offmin[0].size(), offmin[0].empty() ? 0.0 : offmin[0][0],
                offmax[0].empty() ? 0.0 : offmax[0][0], sp.nfft, sp.nffti);
    for (size_t i = 0; i < lines.size(); ++i) std::printf("%s%d", i ? "," : "", lines[i]);
    std::printf("],\"mute_depth_off0\":%.6g",
                offmin[0].empty() ? 0.0 : (double)mute_depth(mute, offmin[0][0]));
    if (check_only >= 2) {
      // dry run of the inputs: every line's tables as a run loads them, and
      // every data file the lines read (whole traces, trailing partial bytes)
      std::printf(",\"tables\":[");
      for (size_t i = 0; i < lines.size(); ++i) {
        Tables tt, tq;
        const bool ht = load_tables(ttpath, false, lines[i], line1, line2, tt);
        const bool hq = ht && load_tables(ttpath, true, lines[i], line1, line2, tq);
        std::printf("%s{\"line\":%d,\"ttt\":%lld,\"qqq\":%lld,\"nxg\":%d,\"nzg\":%d}",
                    i ? "," : "", lines[i], ht ? (long long)tt.data.size() : -1LL,
                    hq ? (long long)tq.data.size() : -1LL, tt.nxg, tt.nzg);
      }
      std::printf("],\"data\":[");
      const size_t rb = kHdr + 4 * (size_t)ntl;
      int nf = 0;
      for (size_t k = 0; k < offmin[0].size(); ++k)
        for (int l = line1; l <= line2; ++l) {
          const std::string f = offspath + "/off" + std::to_string(k) + "/line" + std::to_string(l);
          struct stat st;
          if (stat(f.c_str(), &st) != 0) continue;
          std::printf("%s{\"file\":\"%s\",\"traces\":%lld,\"partial_bytes\":%lld}",
                      nf++ ? "," : "", f.c_str(), (long long)(st.st_size / (long long)rb),
                      (long long)(st.st_size % (long long)rb));
        }
      std::printf("]");
    }
    std::printf("}\n");
    return 0;
  }
  int ngpu = 0;
  if (cudaGetDeviceCount(&ngpu) != cudaSuccess || ngpu <= 0) die("no CUDA device");
  if (igpu >= ngpu) {
    logf("Warn: This Machine [%s] has no such GPU using id=%d instead\n", nodename.c_str(),
         igpu % ngpu);
    igpu %= ngpu;
  }
  std::vector<int> iaz(4096);
  const int naz = qpsdm_build_iaztab(sp.eps, iaz.data(), (int)iaz.size());
  qpsdm_engine *eng = nullptr;
  check_engine(qpsdm_engine_create(&sp, iaz.data(), naz, igpu, &eng), nullptr, "engine create");
  cudaSetDevice(igpu);  // the driver's own device buffers (tables) on the engine's GPU

  // constant dip limits (src/q-psdm.cu:1463-1472): the argument summed in
  // double and rounded to float, then the float tangent
  const size_t nxz = (size_t)nxi * nzi;
  std::vector<float> dx1(nxz, tanf((float)(-10 * 0.0174532925199 + (double)sp.contract)));
  std::vector<float> dx2(nxz, tanf((float)(10 * 0.0174532925199 - (double)sp.contract)));
  const size_t rec_bytes = kHdr + 4 * (size_t)ntl;
  Producer prod(rec_bytes, max_batch, 2);
  const int nxb1 = (int)(nxi / nblock + 0.5);

  // resume after the last finished line
  size_t first = 0;
  if (resume) {
    FILE *fp = std::fopen((offspath + "/break_point.txt").c_str(), "r");
    int done_line;
    if (fp && std::fscanf(fp, "%d", &done_line) == 1)
      for (size_t i = 0; i < lines.size(); ++i)
        if (lines[i] == done_line) first = i + 1;
    if (fp) std::fclose(fp);
    logf("resume: starting at line index %zu\n", first);
  }

  // Lines are imaged `brick` at a time (engine bricks: one pass over the data
  // for all of them; in the batched physics form each trace's t* panels are
  // shared).  Each data-line file feeds only the brick's image lines within
  // +-extxline of it, as the reference's per-line passes do.
  const int16_t vel_scalco = be_i16(v0.h + oScalco);
  std::vector<float> img;
  for (size_t b0 = first; b0 < lines.size(); b0 += brick) {
    const int nl = (int)std::min((size_t)brick, lines.size() - b0);
    const time_t tic = std::time(nullptr);
    std::vector<int> bl(lines.begin() + b0, lines.begin() + b0 + nl);
    std::vector<std::vector<int32_t>> csx(nl, std::vector<int32_t>(nxi)),
        csy(nl, std::vector<int32_t>(nxi));
    std::vector<Tables> tt(nl), tq(nl);
    std::vector<qpsdm_line_params> lps(nl);
    for (int j = 0; j < nl; ++j) {
      const int line = bl[j];
      logf("Start Image Line:%d\n", line);
      // output coordinates from the velocity file (get_vel_coor, src/psdmpkg.cc:979-1011)
      const int vl = std::min(line, flv + nyv - 1);
      for (int i = 0; i < nxi; ++i) {
        TraceHdr t;
        if (!read_header(vf, (long)(vl - flv) * nxv + fci - fcv + i, ntv, t))
          die("velocity file too short for line %d", line);
        csx[j][i] = be_i32(t.h + oSx);
        csy[j][i] = be_i32(t.h + oSy);
      }
      // tables (required in physics mode)
      const bool have_t = load_tables(ttpath, false, line, line1, line2, tt[j]);
      const bool have_q = have_t && load_tables(ttpath, true, line, line1, line2, tq[j]);
      if (sp.mode == QPSDM_MODE_PHYSICS && !(have_t && have_q))
        die("physics mode needs %s/Lxxx.tidx and Lxxx.qidx", ttpath.c_str());
      if (have_q && (tt[j].cdp1 != tq[j].cdp1 || tt[j].cdp2 != tq[j].cdp2 ||
                     tt[j].cdp1 >= tt[j].cdp2))
        die("travel time table cdp range error, or not confirm with qfield");
      qpsdm_line_params &lp = lps[j];
      std::memset(&lp, 0, sizeof lp);
      lp.fxi = fxv + (double)((float)(fci - fcv) * dxi);  // src/q-psdm.cu:1430-1431
      lp.cyi = fyv + (double)((float)(line - flv) * dyi);
      lp.dipx1 = dx1.data();
      lp.dipx2 = dx2.data();
      lp.dipy1 = dx1.data();
      lp.dipy2 = dx2.data();
      if (have_q) {
        lp.nxg = tt[j].nxg;
        lp.nzg = tt[j].nzg;
        lp.nxi1 = tt[j].nxi1;
        lp.nzi1 = tt[j].nzi1;
        lp.ttt_cdp1 = tt[j].cdp1;
        lp.ttt_cdp2 = tt[j].cdp2;
        lp.ttt_desc = tt[j].desc.data();
        lp.qqq_desc = tq[j].desc.data();
        lp.ttt_len = (int64_t)tt[j].data.size();
        lp.qqq_len = (int64_t)tq[j].data.size();
        lp.ttt = tables_on_device(tt[j], line);
        lp.qqq = tables_on_device(tq[j], line);
      }
    }
    check_engine(qpsdm_set_lines(eng, lps.data(), nl), eng, "set_lines");
    // the data lines some image line of the brick reads, and which ones
    // (src/q-psdm.cu:1432-1435: line +- extxline inside [line1, line2])
    std::vector<std::pair<int, unsigned long long>> dlines;
    for (int l = line1; l <= line2; ++l) {
      unsigned long long mask = 0;
      for (int j = 0; j < nl; ++j)
        if (l >= bl[j] - xline && l <= bl[j] + xline) mask |= 1ull << j;
      if (mask) dlines.push_back({l, mask});
    }

    for (int iblock = 0; iblock < nblock; ++iblock) {
      const int ixstart = iblock * nxb1, ixend = iblock == nblock - 1 ? nxi : (iblock + 1) * nxb1;
      const int nxb = ixend - ixstart;
      img.assign((size_t)nl * nxb * nzi, 0.0f);
      for (int id = 0; id < ndata; ++id) {
        const std::string outputpath =
            pp.projpath + "/" + std::to_string(id) + "/" + pp.task + "/result";
        const std::string node_i = node0 + "_" + std::to_string(id);
        offspath = pp.projpath + "/data" + std::to_string(id);
        infopath = pp.projpath + "/" + std::to_string(id) + "/" + pp.task;
        for (size_t k = 0; k < offmin[id].size(); ++k) {
          std::vector<std::string> out(nl);
          for (int j = 0; j < nl; ++j) {
            out[j] = outputpath + "/" + node_i + ".off" + std::to_string(k) + ".L" +
                     std::to_string(bl[j]) + ".su";
            if (iblock == 0 && exists(out[j])) unlink(out[j].c_str());
          }
          float tm = mute_depth(mute, offmin[id][k]);
          if (tm < 0) tm = 0;
          if (tm < zmin) tm = zmin;
          if ((int)(tm / dzi) > nzi) {
            logf("Warn: Offset=%f is greater than the offset mute parameter: no image\n", tm);
            continue;
          }
          qpsdm_offset_params op;
          check_engine(qpsdm_offset_params_init(&sp, ixstart, ixend, &op), eng, "offset params");
          op.ioffs = (int)k;
          for (int a = 0; a < QPSDM_NAZ; ++a) {
            op.aznx1[a] = op.aznx2[a] = aperx;
            op.azny1[a] = op.azny2[a] = apery;
          }
          op.zero_image = opcrp;
          check_engine(qpsdm_begin_offset(eng, &op), eng, "begin_offset");
          std::vector<std::pair<std::string, int>> files;
          for (const auto &d : dlines)
            files.push_back({offspath + "/off" + std::to_string(k) + "/line" +
                                 std::to_string(d.first), d.first});
          prod.start(files);
          int b, n, dl;
          size_t di = 0;
          while (prod.next(b, n, dl)) {
            while (di < dlines.size() && dlines[di].first != dl) ++di;
            if (nl > 1) check_engine(qpsdm_set_line_mask(eng, dlines[di].second), eng, "line mask");
            check_engine(qpsdm_submit_traces(eng, prod.data(b), n, ntl, 1), eng, "submit_traces");
            prod.release(b);
          }
          prod.join();
          if (nl > 1) check_engine(qpsdm_set_line_mask(eng, ~0ull), eng, "line mask");
          if (!opcrp) continue;  // no crp output: the image keeps accumulating
          check_engine(qpsdm_get_image(eng, img.data(), 1), eng, "get_image");
          // append each line's block traces (src/q-psdm.cu:1766-1806)
          mkdir((pp.projpath + "/" + std::to_string(id)).c_str(), 0755);
          mkdir(infopath.c_str(), 0755);
          mkdir(outputpath.c_str(), 0755);
          std::vector<uint8_t> rec(kHdr + 4 * (size_t)nzi);
          for (int j = 0; j < nl; ++j) {
            FILE *fo = std::fopen(out[j].c_str(), "ab");
            if (!fo)
              die("On [%s], File [%s] Open Error: %s", node_i.c_str(), out[j].c_str(),
                  std::strerror(errno));
            int tracl = 0;
            for (int c : cdps) {
              const int ixi = c - cdp1;
              if (ixi < ixstart || ixi >= ixend) continue;
              std::memset(rec.data(), 0, kHdr);
              put_i32(rec.data() + oTracl, ++tracl);
              put_i32(rec.data() + oFldr, bl[j]);
              put_i32(rec.data() + oCdp, fci + ixi);
              put_i16(rec.data() + oTrid, 1);
              put_i16(rec.data() + oNvs, 1);
              put_i32(rec.data() + oOffset, (int32_t)offmin[id][k]);
              put_i16(rec.data() + oScalco, vel_scalco);
              put_i32(rec.data() + oSx, csx[j][ixi]);
              put_i32(rec.data() + oSy, csy[j][ixi]);
              put_i32(rec.data() + oGx, csx[j][ixi]);
              put_i32(rec.data() + oGy, csy[j][ixi]);
              put_i16(rec.data() + oCounit, 1);
              put_i16(rec.data() + oNs, (int16_t)nzi);
              put_i16(rec.data() + oDt, (int16_t)(int)(dzi * 1.0E3f));
              const float *col = img.data() + ((size_t)j * nxb + (ixi - ixstart)) * nzi;
              for (int z = 0; z < nzi; ++z) {
                uint32_t u;
                std::memcpy(&u, col + z, 4);
                put_i32(rec.data() + kHdr + 4 * z, (int32_t)u);
              }
              std::fwrite(rec.data(), 1, rec.size(), fo);
            }
            std::fclose(fo);
            logf("Write Image(crp) To Disk For Line %d:%s\n", bl[j], out[j].c_str());
          }
        }
      }
    }
    // checkpoint markers (src/q-psdm.cu:1820-1831), after each line of the brick
    for (int j = 0; j < nl; ++j) {
      touch(offspath + "/break_point.txt", std::to_string(bl[j]) + "\n");
      touch(infopath + "/" + node0 + "_" + std::to_string(ndata - 1) + "_" +
                std::to_string(bl[j]), "");
    }
    logf("Time Elapse of Lines %d..%d:%.0fs\n", bl.front(), bl.back(),
         std::difftime(std::time(nullptr), tic));
  }
  touch(pp.projpath + "/0/" + pp.task + "/" + node0, "");
  int64_t acc = 0, npt = 0;
  qpsdm_get_counters(eng, &acc, &npt);
  logf("%s: All Migration Work Done (%lld traces accepted, %lld point-traces)\n", nodename.c_str(),
       (long long)acc, (long long)npt);
  qpsdm_engine_destroy(eng);
  std::fclose(vf);
  return 0;
}
