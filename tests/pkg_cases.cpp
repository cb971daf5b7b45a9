// pkg_cases.cpp -- the q-psdm driver's utility API exercised case by case,
// printing a transcript (floats as their bit patterns) that the library must
// reproduce exactly.  Built against this repository's headers and
// libqpsdm_pkg.so, or with -DPKG_REF against the reference's psdmpkg.h /
// segy.h and its compiled psdmpkg.cc / segy.cc (the transcript in
// tests/golden/pkg_cases.txt was made that way).  Only inputs on which the
// reference is well defined are used.  Files are written in the working
// directory.
#ifdef PKG_REF
#include "psdmpkg.h"
// defined in psdmpkg.cc, not declared in its header
int getparstr(const char *key, const char **val);
#else
#include "qpsdm_psdmpkg.h"
#endif

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

uint64_t g_state = 0x9e3779b97f4a7c15ull;
uint32_t rnd() {
  g_state = g_state * 6364136223846793005ull + 1442695040888963407ull;
  return (uint32_t)(g_state >> 33);
}
float rndf() { return (float)((int)(rnd() % 2000001) - 1000000) / 4096.0f; }

uint32_t bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

void hex(const char *tag, const void *p, size_t n) {
  const unsigned char *b = static_cast<const unsigned char *>(p);
  std::printf("%s", tag);
  for (size_t i = 0; i < n; ++i) std::printf("%02x", b[i]);
  std::printf("\n");
}

void floats(const char *tag, const float *v, int n) {
  std::printf("%s n=%d", tag, n);
  for (int i = 0; i < n; ++i) std::printf(" %08x", bits(v[i]));
  std::printf("\n");
}

void write_file(const char *path, const std::string &text) {
  FILE *f = std::fopen(path, "w");
  std::fwrite(text.data(), 1, text.size(), f);
  std::fclose(f);
}

void put_be(unsigned char *p, uint32_t v, int nbytes) {
  for (int i = 0; i < nbytes; ++i) p[i] = (unsigned char)(v >> (8 * (nbytes - 1 - i)));
}

// ---- lists and tuples -------------------------------------------------------
void case_parseint() {
  const char *lists[] = {"5",        "1,3,5",       "1-5",          "2,4-7,9",
                         "1:2:9",    "10:2:31",     "3,1:2:7,20-22", "7-9,1:3:10",
                         "1:2:8-10", "100:25:200,7", "4-4,4",        "0:5:4",
                         "12,13,14,15,16,17", "1:1:1"};
  for (const char *s : lists) {
    int n = -1;
    int *p = parseline(s, &n);
    std::printf("parseint [%s] n=%d:", s, n);
    for (int i = 0; i < n; ++i) std::printf(" %d", p[i]);
    std::printf("\n");
    std::free(p);
  }
}

void case_parsetuple() {
  const char *tuples[] = {"(1,2),(3,4)",
                          "(1.5 2.5 3)(4 5 6)",
                          "(1e3;2),(3,4),(5,6)",
                          "(0,1500),(3000,2500),(6000,3500),(9000,4000)",
                          " ( 10 , 20 ) , ( 30 , 40 ) ",
                          "(1,2),(3)",
                          "(1,2),(3,4",
                          "1,2",
                          "(.5,2.),(7.25,1E2)",
                          "(),()"};
  for (const char *s : tuples) {
    int nt = -1, ne = -1;
    float *p = parsetuple(s, &nt, &ne);
    std::printf("parsetuple [%s] null=%d", s, p == nullptr);
    floats("", p, p ? nt * ne : 0);
    std::printf("  ntuple=%d nelem=%d\n", nt, ne);
    std::free(p);
  }
}

// ---- par.dat ------------------------------------------------------------------
void case_readparfile() {
  std::string long_value(1500, 'x');
  std::string par =
      "# survey parameters\n"
      "   nx=100\n"
      "dx=12.5   # metres\n"
      "\t ny = 7\n"
      "ny=8\n"
      "name=abc def\n"
      "path=/data/run one/out  \n"
      "vel=/data/v.su\n"
      "   # indented comment\n"
      "\n"
      "fmax=60.\\\n"
      "5\n"
      "list=1,2,\\\n"
      "   3,4\n"
      "dup=1\n"
      "dup=2\n"
      "long=" + long_value + "\n" +
      "gval=2.5e-3\n"
      "tail=noeol";
  write_file("case.par", par);

  int nx = -7, ny = -7, d1 = -7, d2 = -7, missing = -7;
  float dx = -7.0f, fmax = -7.0f, g = -7.0f;
  char name[2048] = "unset", vel[2048] = "unset";
  char *path = nullptr, *list = nullptr, *lng = nullptr, *tail = nullptr;

  int r = readparfile("case.par", "nx=%d", &nx);
  std::printf("readpar nx r=%d nx=%d\n", r, nx);
  r = readparfile("case.par", "nx=%d,dx=%f,fmax=%f,gval=%g", &nx, &dx, &fmax, &g);
  std::printf("readpar four r=%d nx=%d dx=%08x fmax=%08x g=%08x\n", r, nx, bits(dx),
              bits(fmax), bits(g));
  r = readparfile("case.par", "ny=%d", &ny);
  std::printf("readpar ny r=%d ny=%d\n", r, ny);
  r = readparfile("case.par", "name=%s,vel=%s", name, vel);
  std::printf("readpar strings r=%d name=[%s] vel=[%s]\n", r, name, vel);
  r = readparfile("case.par", "path=%S,list=%S", &path, &list);
  std::printf("readpar rest r=%d path=[%s] list=[%s]\n", r, path ? path : "(null)",
              list ? list : "(null)");
  std::free(path);
  std::free(list);
  r = readparfile("case.par", "dup=%d,nx=%d", &d1, &d2);
  std::printf("readpar dup r=%d d1=%d d2=%d\n", r, d1, d2);
  r = readparfile("case.par", "missing=%d", &missing);
  std::printf("readpar missing r=%d v=%d\n", r, missing);
  r = readparfile("case.par", "long=%S", &lng);
  std::printf("readpar long r=%d len=%zu\n", r, lng ? std::strlen(lng) : (size_t)0);
  std::free(lng);
  r = readparfile("case.par", "tail=%S", &tail);
  std::printf("readpar tail r=%d tail=%s\n", r, tail ? "set" : "(null)");
  std::free(tail);
}

// ---- command line -------------------------------------------------------------
void case_getpar() {
  const char *argv0[] = {"q-psdm", "nx=240",  "n=5",        "dx=12.5e0", "path=/a/b=c",
                         "nx=999", "fmax=60", "eps=1e-30", "neg=-17",   "dt=0.004",
                         "flag="};
  std::vector<char *> argv;
  for (const char *a : argv0) argv.push_back(const_cast<char *>(a));
  initargs_inner((int)argv.size(), argv.data(), nullptr);
  std::printf("initargs xargc=%d last=[%s]\n", xargc, xargv[xargc - 1]);
  int i = -1, r;
  r = getparint("nx", &i);
  std::printf("getparint nx r=%d v=%d\n", r, i);
  r = getparint("n", &i);
  std::printf("getparint n r=%d v=%d\n", r, i);
  r = getparint("neg", &i);
  std::printf("getparint neg r=%d v=%d\n", r, i);
  i = -1;
  r = getparint("ny", &i);
  std::printf("getparint ny r=%d v=%d\n", r, i);
  float f = -1.0f;
  r = getparfloat("dx", &f);
  std::printf("getparfloat dx r=%d v=%08x\n", r, bits(f));
  r = getparfloat("eps", &f);
  std::printf("getparfloat eps r=%d v=%08x\n", r, bits(f));
  r = getparfloat("dt", &f);
  std::printf("getparfloat dt r=%d v=%08x\n", r, bits(f));
  double d = -1.0;
  r = getpardouble("dt", &d);
  std::printf("getpardouble dt r=%d v=%.17g\n", r, d);
  char *s = nullptr;
  r = getparstring("path", &s);
  std::printf("getparstr path r=%d v=[%s]\n", r, s ? s : "(null)");
  const char *cs = nullptr;
  r = getparstring("flag", &cs);
  std::printf("getparstr flag r=%d v=[%s]\n", r, cs ? cs : "(null)");
  cs = nullptr;
  r = getparstring("pat", &cs);
  std::printf("getparstr pat r=%d null=%d\n", r, cs == nullptr);
}

// ---- taper, mute, scale, paths -------------------------------------------------
void case_taper() {
  std::vector<float> data(1000);
  for (float &v : data) v = rndf();
  const int windows[][2] = {{-50, 600}, {100, 1100}, {0, 150}, {400, 999}, {-10, 1010},
                            {500, 500}};
  for (const auto &w : windows) {
    std::vector<float> out(w[1] - w[0] + 1, -1.0f);
    const int r = fetch_and_taper(data.data(), 1000, w[0], w[1], out.data());
    char tag[64];
    std::snprintf(tag, sizeof tag, "taper [%d,%d] r=%d", w[0], w[1], r);
    floats(tag, out.data(), (int)out.size());
  }
}

void case_mute() {
  std::vector<std::vector<float>> sets = {
      {0.0f, 0.0f, 500.0f, 1000.0f, 1500.0f, 3000.0f},
      {100.0f, 0.0f, 80.0f, 500.0f, 300.0f, 400.0f, 300.0f, 2000.0f},
      {200.0f, 100.0f, 200.0f, 100.0f, 200.0f, 100.0f},
      {0.1f, 0.3f, 0.7f, 0.2f, 1.9f, 3.1f},
      {800.0f, 1200.0f}};
  const float offs[] = {-500.0f, 0.0f, 250.0f, 999.5f, 1000.0f, 2999.0f, 3000.0f, 7000.0f};
  for (auto &m : sets) {
    const int n = (int)m.size() / 2;
    floats("mute in", m.data(), 2 * n);
    time_offset_mute_santity(m.data(), n);
    floats("mute sane", m.data(), 2 * n);
    for (float o : offs)
      std::printf("mute n=%d o=%08x t=%08x\n", n, bits(o), bits(time_offset_mute(m.data(), n, o)));
  }
}

void case_scale_paths() {
  const short sc[] = {0, 1, 10, -1, -10, -100, 1000, -1000, 32767, -32768, 3, -3, -7};
  for (short s : sc) std::printf("getscale %d %08x\n", s, bits(getscale(s)));

  const char *paths[] = {"/data/proj/myproj/3/task1", "proj/12/t", "/x/1/imaging",
                         "base/root/7/migrate.job"};
  for (const char *p0 : paths) {
    char path[256], projpath[256] = "", projname[256] = "", task[256] = "";
    std::strcpy(path, p0);
    int iproc = -1;
    parsepath(path, projpath, projname, &iproc, task);
    std::printf("parsepath [%s] projpath=[%s] projname=[%s] iproc=%d task=[%s]\n", p0,
                projpath, projname, iproc, task);
  }

  const char *trims[] = {"abc///", "abc", "a/b/", "xx"};
  for (const char *t : trims) {
    char b[64];
    std::strcpy(b, t);
    std::printf("strrtrim [%s] -> [%s]\n", t, strrtrim(b, '/'));
  }

  write_file("size.bin", std::string(12345, 'q'));
  std::printf("fsize %zu exist %d %d\n", fsize("size.bin"), exist("size.bin"),
              exist("no-such-file.bin"));
}

// ---- SU records -----------------------------------------------------------------
void random_record(std::vector<unsigned char> &rec, int ns) {
  rec.assign(240 + 4 * (size_t)ns, 0);
  for (int i = 0; i < 240; ++i) rec[i] = (unsigned char)rnd();
  put_be(&rec[114], (uint32_t)ns, 2);  // ns, big-endian
  for (int i = 0; i < ns; ++i) put_be(&rec[240 + 4 * i], bits(rndf()), 4);
}

void case_segy() {
  segy *tr = static_cast<segy *>(std::malloc(sizeof(segy)));
  // reading: a file of random headers
  const int nss[] = {37, 1, 256, 1000};
  {
    FILE *f = std::fopen("rand.su", "wb");
    std::vector<unsigned char> rec;
    for (int ns : nss) {
      random_record(rec, ns);
      std::fwrite(rec.data(), 1, rec.size(), f);
    }
    rec.resize(240 + 4 * 10);  // a record cut short
    random_record(rec, 64);
    std::fwrite(rec.data(), 1, 240 + 4 * 10, f);
    std::fclose(f);
  }
  FILE *f = std::fopen("rand.su", "rb");
  for (int k = 0; k < 6; ++k) {
    std::memset(tr, 0xa5, sizeof(segy));
    const int ns = fgettr(f, tr);
    std::printf("fgettr %d ns=%d\n", k, ns);
    if (ns > 0) {
      hex("fgettr hdr ", tr, 240);
      floats("fgettr data", tr->data, ns);
    }
  }
  std::fclose(f);

  // sgettr from memory
  for (int ns : nss) {
    std::vector<unsigned char> rec;
    random_record(rec, ns);
    std::memset(tr, 0x5a, sizeof(segy));
    const int r = sgettr(rec.data(), tr);
    std::printf("sgettr ns=%d r=%d\n", ns, r);
    hex("sgettr hdr ", tr, 240);
    floats("sgettr data", tr->data, ns);
  }

  // writing: random headers in native order
  f = std::fopen("out.su", "wb");
  for (int ns : nss) {
    unsigned char *h = reinterpret_cast<unsigned char *>(tr);
    for (int i = 0; i < 240; ++i) h[i] = (unsigned char)rnd();
    tr->ns = (unsigned short)ns;
    for (int i = 0; i < ns; ++i) tr->data[i] = rndf();
    fputtr(f, tr);
    std::vector<unsigned char> buf(240 + 4 * (size_t)ns, 0xcc);
    sputtr(buf.data(), tr);
    hex("sputtr hdr ", buf.data(), 240);
    hex("sputtr data ", buf.data() + 240, 4 * (size_t)ns);
  }
  std::fclose(f);
  f = std::fopen("out.su", "rb");
  std::vector<unsigned char> all;
  unsigned char c[4096];
  size_t got;
  while ((got = std::fread(c, 1, sizeof c, f)) > 0) all.insert(all.end(), c, c + got);
  std::fclose(f);
  std::printf("fputtr bytes=%zu\n", all.size());
  size_t off = 0;
  for (int ns : nss) {
    hex("fputtr hdr ", all.data() + off, 240);
    hex("fputtr data ", all.data() + off + 240, 4 * (size_t)ns);
    off += 240 + 4 * (size_t)ns;
  }
  std::free(tr);
}

void case_vel_coor() {
  // a velocity file of nyv lines x nxv cdps, 50 samples, coordinates by position
  const int nxv = 30, nyv = 6, flv = 100, fcv = 200, ns = 50;
  segy *tr = static_cast<segy *>(std::malloc(sizeof(segy)));
  std::memset(tr, 0, sizeof(segy));
  FILE *f = std::fopen("vel.su", "wb");
  for (int y = 0; y < nyv; ++y)
    for (int x = 0; x < nxv; ++x) {
      tr->ns = ns;
      tr->scalco = -100;
      tr->sx = 1000000 + 2500 * x + 7 * y;
      tr->sy = 5000000 + 2500 * y + 3 * x;
      tr->cdp = fcv + x;
      for (int i = 0; i < ns; ++i) tr->data[i] = 1500.0f + i;
      fputtr(f, tr);
    }
  std::fclose(f);
  std::free(tr);
  const int cases[][3] = {{100, 200, 30}, {102, 205, 10}, {105, 229, 1}, {109, 210, 5}};
  for (const auto &c : cases) {
    std::vector<coor_t> co(c[2]);
    short sc = 0;
    get_vel_coor("vel.su", c[0], co.data(), &sc, c[1], c[2], fcv, nxv, flv, nyv);
    std::printf("get_vel_coor line=%d fci=%d nxi=%d scalco=%d:", c[0], c[1], c[2], sc);
    for (const coor_t &p : co) std::printf(" %d,%d", p.sx, p.sy);
    std::printf("\n");
  }
}

void case_arrays() {
  float **a = alloc2float(7, 5);
  int **b = alloc2int(3, 4);
  char **c = alloc2char(11, 2);
  std::printf("arrays rows %td %td %td\n", a[4] - a[0], b[3] - b[0], c[1] - c[0]);
  free2float(a);
  free2int(b);
  free2char(c);
}

}  // namespace

int main() {
  case_parseint();
  case_parsetuple();
  case_readparfile();
  case_getpar();
  case_taper();
  case_mute();
  case_scale_paths();
  case_segy();
  case_vel_coor();
  case_arrays();
  return 0;
}
