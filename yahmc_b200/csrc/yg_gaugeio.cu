// Gauge configuration files: the native CFG format (gaugefield.cpp:44-179) and the HiRep
// format (hirep.cpp:56-212).  Both store, for t, x, y, z in lexicographic order, the four
// fundamental links of the site as N*N (re, im) double pairs (suNg::write, suNg.cpp:392-412);
// CFG starts with a packed 256-byte header in the machine's byte order, HiRep with five
// big-endian ints (N, T, X, Y, Z) and a big-endian plaquette, and stores its doubles
// big-endian.  The whole file is assembled in host memory and moved in one read or write;
// the links go to and from the device in the reference's host layout.  Loading applies the
// gauge boundary conditions and represents the field, as the reference does.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "yg_lattice.h"

namespace yg {

namespace {

constexpr int kCfgIdent = 0x47464359, kCfgVersion = 0x20;   // include/gaugefield.h:20-21

#pragma pack(push, 1)
struct CfgHeader {          // header_t, include/gaugefield.h:23-36
  int32_t ident, version, dim_t, dim_x, dim_y, dim_z, nc, repr, num_cnfg, num_accept;
  double plaquette;
  char reserved[208];
};
#pragma pack(pop)
static_assert(sizeof(CfgHeader) == 256, "CFG header is 256 bytes");

template <typename T>
T swap_bytes(T v) {
  unsigned char b[sizeof(T)];
  std::memcpy(b, &v, sizeof(T));
  for (size_t i = 0; i < sizeof(T) / 2; i++) std::swap(b[i], b[sizeof(T) - 1 - i]);
  std::memcpy(&v, b, sizeof(T));
  return v;
}

// the even-odd site id of lexicographic position lex (geometry.cpp ordering with UPDATE_EO)
long site_of_lex(const Lattice &L, long lex) {
  const int *d = L.p.dims;
  if (!L.p.eo) return lex;
  long r = lex;
  const int z = (int)(r % d[3]); r /= d[3];
  const int y = (int)(r % d[2]); r /= d[2];
  const int x = (int)(r % d[1]);
  const int t = (int)(r / d[1]);
  const int p = (t + x + y + z) & 1;
  return (p * L.V + lex) / 2;
}

// host layout <-> file body.  Host: links[(4*id + mu)] as {re[N*N], im[N*N]}; file: per site
// in lexicographic order, per mu, the N*N (re, im) pairs.
void to_file(const Lattice &L, const std::vector<double> &host, std::vector<double> &body, bool big_endian) {
  const int nn = L.nc * L.nc;
  body.resize((size_t)L.V * 4 * 2 * nn);
  size_t o = 0;
  for (long lex = 0; lex < L.V; lex++) {
    const long id = site_of_lex(L, lex);
    for (int mu = 0; mu < 4; mu++) {
      const double *rec = host.data() + (size_t)(4 * id + mu) * 2 * nn;
      for (int k = 0; k < nn; k++) {
        double re = rec[k], im = rec[nn + k];
        if (big_endian) { re = swap_bytes(re); im = swap_bytes(im); }
        body[o++] = re;
        body[o++] = im;
      }
    }
  }
}

void from_file(const Lattice &L, const std::vector<double> &body, std::vector<double> &host, bool big_endian) {
  const int nn = L.nc * L.nc;
  host.resize((size_t)L.V * 4 * 2 * nn);
  size_t o = 0;
  for (long lex = 0; lex < L.V; lex++) {
    const long id = site_of_lex(L, lex);
    for (int mu = 0; mu < 4; mu++) {
      double *rec = host.data() + (size_t)(4 * id + mu) * 2 * nn;
      for (int k = 0; k < nn; k++) {
        double re = body[o++], im = body[o++];
        if (big_endian) { re = swap_bytes(re); im = swap_bytes(im); }
        rec[k] = re;
        rec[nn + k] = im;
      }
    }
  }
}

struct File {
  FILE *f;
  File(const char *path, const char *mode) : f(std::fopen(path, mode)) {
    if (!f) throw Error(YG_ERR_ARG, std::string("unable to open file: ") + path);
  }
  ~File() { if (f) std::fclose(f); }
  void write(const void *p, size_t n) {
    if (std::fwrite(p, 1, n, f) != n) throw Error(YG_ERR_ARG, "short write");
  }
  void read(void *p, size_t n) {
    if (std::fread(p, 1, n, f) != n) throw Error(YG_ERR_ARG, "file shorter than the configuration it describes");
  }
};

}  // namespace

// gauge_field_save, gaugefield.cpp:44-106 (the reserved header bytes are written as zeros)
void gauge_save_cfg(Lattice &L, const char *path, int num_cnfg, int num_accept) {
  CfgHeader h;
  std::memset(&h, 0, sizeof(h));
  h.ident = kCfgIdent;
  h.version = kCfgVersion;
  h.dim_t = L.p.dims[0]; h.dim_x = L.p.dims[1]; h.dim_y = L.p.dims[2]; h.dim_z = L.p.dims[3];
  h.nc = L.nc;
  h.repr = L.p.repr;
  h.num_cnfg = num_cnfg;
  h.num_accept = num_accept;
  h.plaquette = avr_plaquette(L);
  std::vector<double> host((size_t)L.V * 4 * 2 * L.nc * L.nc), body;
  gauge_download(L, host.data());
  to_file(L, host, body, false);
  File f(path, "wb");
  f.write(&h, sizeof(h));
  f.write(body.data(), body.size() * sizeof(double));
}

// gauge_field_load, gaugefield.cpp:108-161: an inconsistent header is an error (the
// reference stops); *plaq_diff = |stored plaquette - plaquette of the loaded field|
void gauge_load_cfg(Lattice &L, const char *path, int *num_cnfg, int *num_accept, double *plaq_diff) {
  File f(path, "rb");
  CfgHeader h;
  f.read(&h, sizeof(h));
  int bad = (h.ident != kCfgIdent) + (h.version != kCfgVersion) + (h.dim_t != L.p.dims[0]) +
            (h.dim_x != L.p.dims[1]) + (h.dim_y != L.p.dims[2]) + (h.dim_z != L.p.dims[3]) + (h.nc != L.nc) +
            (h.repr != L.p.repr);
  if (bad) throw Error(YG_ERR_ARG, std::string("configuration is not consistent with the lattice: ") + path);
  std::vector<double> body((size_t)L.V * 4 * 2 * L.nc * L.nc), host;
  f.read(body.data(), body.size() * sizeof(double));
  from_file(L, body, host, false);
  gauge_upload_with_bcs(L, host.data());
  if (num_cnfg) *num_cnfg = h.num_cnfg;
  if (num_accept) *num_accept = h.num_accept;
  if (plaq_diff) *plaq_diff = std::fabs(h.plaquette - avr_plaquette(L));
}

// gauge_field_save_hirep, hirep.cpp:141-212
void gauge_save_hirep(Lattice &L, const char *path) {
  int32_t info[5] = {L.nc, L.p.dims[0], L.p.dims[1], L.p.dims[2], L.p.dims[3]};
  for (int32_t &v : info) v = swap_bytes(v);
  const double plaq = swap_bytes(avr_plaquette(L));
  std::vector<double> host((size_t)L.V * 4 * 2 * L.nc * L.nc), body;
  gauge_download(L, host.data());
  to_file(L, host, body, true);
  File f(path, "wb");
  f.write(info, sizeof(info));
  f.write(&plaq, sizeof(plaq));
  f.write(body.data(), body.size() * sizeof(double));
}

// gauge_field_load_hirep, hirep.cpp:56-139: the configuration number is the integer after
// the last 'n' of the file name (0 if there is none)
void gauge_load_hirep(Lattice &L, const char *path, int *num_cnfg, double *plaq_diff) {
  File f(path, "rb");
  int32_t info[5];
  double plaq;
  f.read(info, sizeof(info));
  f.read(&plaq, sizeof(plaq));
  for (int32_t &v : info) v = swap_bytes(v);
  plaq = swap_bytes(plaq);
  int bad = (info[0] != L.nc) + (info[1] != L.p.dims[0]) + (info[2] != L.p.dims[1]) + (info[3] != L.p.dims[2]) +
            (info[4] != L.p.dims[3]);
  if (bad) throw Error(YG_ERR_ARG, std::string("configuration is not consistent with the lattice: ") + path);
  std::vector<double> body((size_t)L.V * 4 * 2 * L.nc * L.nc), host;
  f.read(body.data(), body.size() * sizeof(double));
  from_file(L, body, host, true);
  gauge_upload_with_bcs(L, host.data());
  if (num_cnfg) {
    *num_cnfg = 0;
    const char *n = std::strrchr(path, 'n');
    if (n) std::sscanf(n, "n%d", num_cnfg);
  }
  if (plaq_diff) *plaq_diff = std::fabs(plaq - avr_plaquette(L));
}

}  // namespace yg
