// NetCDF classic restart files (see rkb_netcdf.hpp).  The encoding follows
// the published NetCDF classic format specification: big-endian header of
// dimensions, global attributes and variables (name, dimension ids,
// attributes, type, size, data offset), then each fixed-size variable's
// values contiguous at its offset, padded to 4 bytes.
#include "rkb_netcdf.hpp"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace rkb {
namespace nc {
namespace {

constexpr uint32_t kDimTag = 0x0A, kVarTag = 0x0B, kAttTag = 0x0C;
constexpr uint32_t kChar = 2, kShort = 3, kInt = 4, kFloat = 5, kDouble = 6, kByte = 1;

uint32_t pad4(uint32_t n) { return (n + 3u) & ~3u; }
uint64_t pad4_64(uint64_t n) { return (n + 3ull) & ~3ull; }

// ---- writer -----------------------------------------------------------------

struct Out {
  std::vector<unsigned char> b;
  void u32(uint32_t v) {
    for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
  }
  void u64(uint64_t v) {
    for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
  }
  void name(const std::string& s) {
    u32((uint32_t)s.size());
    b.insert(b.end(), s.begin(), s.end());
    while (b.size() % 4) b.push_back(0);
  }
  void text_att(const std::string& n, const std::string& v) {
    name(n);
    u32(kChar);
    u32((uint32_t)v.size());
    b.insert(b.end(), v.begin(), v.end());
    while (b.size() % 4) b.push_back(0);
  }
  void double_att(const std::string& n, double v) {
    name(n);
    u32(kDouble);
    u32(1);
    uint64_t u;
    std::memcpy(&u, &v, 8);
    u64(u);
  }
  void int_att(const std::string& n, int v) {
    name(n);
    u32(kInt);
    u32(1);
    u32((uint32_t)v);
  }
};

// A global attribute: text, one NC_DOUBLE or one NC_INT.
struct Att {
  std::string name;
  uint32_t type;
  std::string text;
  double d = 0.0;
  int i = 0;
  Att(std::string n, const char* v) : name(std::move(n)), type(kChar), text(v) {}
  Att(std::string n, double v) : name(std::move(n)), type(kDouble), d(v) {}
  Att(std::string n, int v) : name(std::move(n)), type(kInt), i(v) {}
};

void put_be_doubles(std::vector<unsigned char>& dst, const double* v, size_t n) {
  const size_t o = dst.size();
  dst.resize(o + 8 * n);
  for (size_t k = 0; k < n; ++k) {
    uint64_t u;
    std::memcpy(&u, &v[k], 8);
    for (int s = 0; s < 8; ++s) dst[o + 8 * k + s] = (unsigned char)(u >> (56 - 8 * s));
  }
}

std::string num(double x) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.17g", x);
  return buf;
}

// ---- reader -----------------------------------------------------------------

struct In {
  const unsigned char* p;
  size_t n, o = 0;
  bool ok = true;
  uint32_t u32() {
    if (o + 4 > n) { ok = false; return 0; }
    const uint32_t v = (uint32_t)p[o] << 24 | (uint32_t)p[o + 1] << 16 | (uint32_t)p[o + 2] << 8 |
                       (uint32_t)p[o + 3];
    o += 4;
    return v;
  }
  uint64_t u64() {
    const uint64_t hi = u32();
    return hi << 32 | u32();
  }
  std::string name() {
    const uint32_t len = u32();
    if (!ok || o + pad4(len) > n) { ok = false; return {}; }
    std::string s((const char*)p + o, len);
    o += pad4(len);
    return s;
  }
  void skip_atts() {
    const uint32_t tag = u32(), cnt = u32();
    if (tag == 0 && cnt == 0) return;
    if (tag != kAttTag) { ok = false; return; }
    for (uint32_t a = 0; a < cnt && ok; ++a) {
      name();
      const uint32_t type = u32(), nel = u32();
      const uint32_t sz = type == kByte || type == kChar ? 1 : type == kShort ? 2 :
                          type == kDouble ? 8 : 4;
      const uint64_t bytes = pad4_64((uint64_t)nel * sz);
      if (o + bytes > n) { ok = false; return; }
      o += bytes;
    }
  }
};

struct Var {
  std::string name;
  std::vector<uint32_t> dims;
  uint32_t type = 0;
  uint64_t begin = 0;
};

}  // namespace

bool write_restart(const std::string& path, int nx, int ny, const double* h, const double* hu,
                   const double* hv, const double* b, double time, double dx, double dy, int ng,
                   std::string& err) {
  const uint64_t n2 = (uint64_t)nx * (uint64_t)ny;
  if (8 * n2 >= 0xFFFFFFFCull) {
    err = "grid too large for a 64-bit-offset NetCDF variable (4 GiB each)";
    return false;
  }
  // header with placeholder offsets, patched once its size is known
  Out hd;
  hd.b = {'C', 'D', 'F', 2};
  hd.u32(0);  // numrecs
  hd.u32(kDimTag);
  hd.u32(2);
  hd.name("x");
  hd.u32((uint32_t)nx);
  hd.name("y");
  hd.u32((uint32_t)ny);
  hd.u32(kAttTag);
  hd.u32(6);
  hd.text_att("Conventions", "CF-1.11");
  hd.text_att("title", "Tidal restart file");
  hd.text_att("source", "rakali_b200");
  hd.text_att("dx", num(dx));
  hd.text_att("dy", num(dy));
  hd.text_att("nghost", std::to_string(ng));
  hd.u32(kVarTag);
  hd.u32(5);
  const char* names[5] = {"h", "hu", "hv", "b", "time"};
  const char* units[5] = {"m", "m2 s-1", "m2 s-1", "m", "seconds since simulation start"};
  size_t begin_at[5];
  for (int v = 0; v < 5; ++v) {
    hd.name(names[v]);
    if (v < 4) {
      hd.u32(2);
      hd.u32(1);  // y (slowest)
      hd.u32(0);  // x
    } else {
      hd.u32(0);
    }
    hd.u32(kAttTag);
    hd.u32(1);
    hd.text_att("units", units[v]);
    hd.u32(kDouble);
    hd.u32(v < 4 ? (uint32_t)(8 * n2) : 8u);
    begin_at[v] = hd.b.size();
    hd.u64(0);
  }
  uint64_t off = hd.b.size();
  for (int v = 0; v < 5; ++v) {
    for (int s = 0; s < 8; ++s) hd.b[begin_at[v] + s] = (unsigned char)(off >> (56 - 8 * s));
    off += v < 4 ? 8 * n2 : 8;
  }
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot open " + path + " for writing";
    return false;
  }
  bool ok = std::fwrite(hd.b.data(), 1, hd.b.size(), f) == hd.b.size();
  std::vector<unsigned char> buf;
  const double* fields[4] = {h, hu, hv, b};
  for (int v = 0; v < 4 && ok; ++v) {
    buf.clear();
    put_be_doubles(buf, fields[v], n2);
    ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  }
  if (ok) {
    buf.clear();
    put_be_doubles(buf, &time, 1);
    ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) err = "write to " + path + " failed";
  return ok;
}

namespace {

// A fixed-size variable to write: dimension ids (slowest first), text
// attributes, and its values (FP64, or characters for NC_CHAR).
struct OutVar {
  std::string name;
  std::vector<uint32_t> dims;
  uint32_t type;
  std::vector<std::pair<std::string, std::string>> atts;
  const void* data;
  uint64_t count;
};

bool write_classic(const std::string& path,
                   const std::vector<std::pair<std::string, uint32_t>>& dims,
                   const std::vector<Att>& gatts, const std::vector<OutVar>& vars,
                   std::string& err) {
  Out hd;
  hd.b = {'C', 'D', 'F', 2};
  hd.u32(0);
  hd.u32(kDimTag);
  hd.u32((uint32_t)dims.size());
  for (const auto& d : dims) {
    hd.name(d.first);
    hd.u32(d.second);
  }
  if (gatts.empty()) {
    hd.u32(0);
    hd.u32(0);
  } else {
    hd.u32(kAttTag);
    hd.u32((uint32_t)gatts.size());
    for (const Att& a : gatts) {
      if (a.type == kDouble)
        hd.double_att(a.name, a.d);
      else if (a.type == kInt)
        hd.int_att(a.name, a.i);
      else
        hd.text_att(a.name, a.text);
    }
  }
  hd.u32(kVarTag);
  hd.u32((uint32_t)vars.size());
  std::vector<size_t> begin_at;
  std::vector<uint64_t> sizes;
  for (const OutVar& v : vars) {
    hd.name(v.name);
    hd.u32((uint32_t)v.dims.size());
    for (uint32_t d : v.dims) hd.u32(d);
    if (v.atts.empty()) {
      hd.u32(0);
      hd.u32(0);
    } else {
      hd.u32(kAttTag);
      hd.u32((uint32_t)v.atts.size());
      for (const auto& a : v.atts) hd.text_att(a.first, a.second);
    }
    hd.u32(v.type);
    // sizes in 64 bits: a 64-bit-offset file stores each variable's size in
    // 32 bits, so anything from 4 GiB - 4 on is refused before narrowing
    const uint64_t sz = pad4_64((uint64_t)v.count * (v.type == kChar ? 1u : 8u));
    if (sz >= 0xFFFFFFFCull) {
      err = "variable " + v.name + " too large for a 64-bit-offset NetCDF file";
      return false;
    }
    hd.u32((uint32_t)sz);
    sizes.push_back(sz);
    begin_at.push_back(hd.b.size());
    hd.u64(0);
  }
  uint64_t off = hd.b.size();
  for (size_t v = 0; v < vars.size(); ++v) {
    for (int s = 0; s < 8; ++s) hd.b[begin_at[v] + s] = (unsigned char)(off >> (56 - 8 * s));
    off += sizes[v];
  }
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot open " + path + " for writing";
    return false;
  }
  bool ok = std::fwrite(hd.b.data(), 1, hd.b.size(), f) == hd.b.size();
  std::vector<unsigned char> buf;
  for (size_t v = 0; v < vars.size() && ok; ++v) {
    buf.clear();
    if (vars[v].type == kChar) {
      const unsigned char* c = (const unsigned char*)vars[v].data;
      buf.assign(c, c + vars[v].count);
    } else {
      put_be_doubles(buf, (const double*)vars[v].data, vars[v].count);
    }
    buf.resize(sizes[v], 0);
    ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) err = "write to " + path + " failed";
  return ok;
}

}  // namespace

bool write_gauges(const std::string& path, int n, const char* names, int name_len,
                  const double* x, const double* y, const double* b, int n_records,
                  const double* times, const double* values, std::string& err) {
  constexpr int kNameLen = 64;  // MAX_NAME_LEN, rki_gauges.F90:26
  std::vector<char> nm((size_t)n * kNameLen, '\0');
  for (int k = 0; k < n; ++k)
    for (int c = 0; c < name_len && c < kNameLen; ++c) {
      const char ch = names ? names[(size_t)k * name_len + c] : '\0';
      if (ch == '\0') break;
      nm[(size_t)k * kNameLen + c] = ch;
    }
  const uint64_t K = (uint64_t)n_records;
  std::vector<double> eta(K * n), u(K * n), v(K * n);
  for (uint64_t r = 0; r < K * n; ++r) {
    eta[r] = values[3 * r];
    u[r] = values[3 * r + 1];
    v[r] = values[3 * r + 2];
  }
  // dimension ids: 0 station, 1 time, 2 name_strlen
  const std::vector<std::pair<std::string, uint32_t>> dims = {
      {"station", (uint32_t)n}, {"time", (uint32_t)n_records}, {"name_strlen", kNameLen}};
  using A = std::vector<std::pair<std::string, std::string>>;
  const std::vector<OutVar> vars = {
      {"time", {1}, kDouble, A{{"units", "seconds"}, {"calendar", "proleptic_gregorian"}}, times, K},
      {"station_name", {0, 2}, kChar, A{}, nm.data(), (uint64_t)n * kNameLen},
      {"station_x", {0}, kDouble, A{{"units", "m"}, {"long_name", "gauge x-coordinate"}}, x,
       (uint64_t)n},
      {"station_y", {0}, kDouble, A{{"units", "m"}, {"long_name", "gauge y-coordinate"}}, y,
       (uint64_t)n},
      {"station_b", {0}, kDouble,
       A{{"units", "m"}, {"long_name", "interpolated bottom elevation"}}, b, (uint64_t)n},
      {"eta", {1, 0}, kDouble, A{{"units", "m"}, {"long_name", "water surface elevation"}},
       eta.data(), K * n},
      {"u", {1, 0}, kDouble, A{{"units", "m/s"}, {"long_name", "depth-averaged x-velocity"}},
       u.data(), K * n},
      {"v", {1, 0}, kDouble, A{{"units", "m/s"}, {"long_name", "depth-averaged y-velocity"}},
       v.data(), K * n}};
  return write_classic(path, dims, {{"title", "Rakali gauge time series"}, {"Conventions", "CF-1.8"}},
                       vars, err);
}

bool write_checkpoint(const std::string& path, int nxt, int nyt, const double* const fields[7],
                      const CheckpointMeta& m, std::string& err) {
  // the file's (x_total, y_total) order has y fastest: the transpose of the
  // Fortran-order arrays
  const size_t n = (size_t)nxt * (size_t)nyt;
  if ((uint64_t)n * 8u >= 0xFFFFFFFCull) {  // checked before the fields are read
    err = "checkpoint fields of " + std::to_string(nxt) + " x " + std::to_string(nyt) +
          " cells are too large for a 64-bit-offset NetCDF file";
    return false;
  }
  std::vector<std::vector<double>> t(7, std::vector<double>(n));
  for (int v = 0; v < 7; ++v)
    for (int j = 0; j < nyt; ++j)
      for (int i = 0; i < nxt; ++i)
        t[v][(size_t)i * nyt + j] = fields[v][(size_t)i + (size_t)j * nxt];
  using A = std::vector<std::pair<std::string, std::string>>;
  const A depth{{"units", "m"}, {"long_name", "water depth (ghost-included)"}};
  const A qx{{"units", "m2 s-1"}, {"long_name", "x-momentum (ghost-included)"}};
  const A qy{{"units", "m2 s-1"}, {"long_name", "y-momentum (ghost-included)"}};
  const A bed{{"units", "m"}, {"long_name", "bottom elevation"}, {"positive", "up"}};
  const A h0{{"units", "m"}, {"long_name", "RK2 save of h at start of stage 1"}};
  const A hu0{{"units", "m2 s-1"}, {"long_name", "RK2 save of hu at start of stage 1"}};
  const A hv0{{"units", "m2 s-1"}, {"long_name", "RK2 save of hv at start of stage 1"}};
  const std::vector<OutVar> vars = {
      {"h", {0, 1}, kDouble, depth, t[0].data(), n}, {"hu", {0, 1}, kDouble, qx, t[1].data(), n},
      {"hv", {0, 1}, kDouble, qy, t[2].data(), n},   {"b", {0, 1}, kDouble, bed, t[3].data(), n},
      {"h0", {0, 1}, kDouble, h0, t[4].data(), n},   {"hu0", {0, 1}, kDouble, hu0, t[5].data(), n},
      {"hv0", {0, 1}, kDouble, hv0, t[6].data(), n}};
  const std::vector<Att> gatts = {{"title", "Rakali per-step checkpoint (2D barotropic)"},
                                  {"source", "rakali_b200 (Rakali.save_checkpoint)"},
                                  {"time", m.time},
                                  {"step_count", m.step_count},
                                  {"dt", m.dt},
                                  {"nx_total", nxt},
                                  {"ny_total", nyt},
                                  {"nx_phys", m.nx_phys},
                                  {"ny_phys", m.ny_phys},
                                  {"nghost", m.nghost},
                                  {"dx", m.dx},
                                  {"dy", m.dy},
                                  {"manning_n", m.manning_n},
                                  {"coriolis_f", m.coriolis_f},
                                  {"clamped_elevation", m.clamped_elevation}};
  return write_classic(path, {{"x_total", (uint32_t)nxt}, {"y_total", (uint32_t)nyt}}, gatts, vars,
                       err);
}

namespace {

// A whole classic file: its dimensions, its variables and the raw bytes.
struct File {
  std::vector<unsigned char> data;
  std::vector<std::pair<std::string, uint32_t>> dims;
  std::vector<Var> vars;

  int dim(const char* nm) const {
    for (size_t d = 0; d < dims.size(); ++d)
      if (dims[d].first == nm) return (int)d;
    return -1;
  }
  const Var* var(const char* nm) const {
    for (const Var& v : vars)
      if (v.name == nm) return &v;
    return nullptr;
  }
  // count values of v (FP64 or FP32 in the file) into dst as doubles
  bool values(const Var& v, uint64_t count, double* dst, std::string& err) const {
    if (v.type != kDouble && v.type != kFloat) {
      err = "variable " + v.name + " is neither double nor float";
      return false;
    }
    const uint64_t sz = v.type == kDouble ? 8 : 4;
    if (v.begin + sz * count > data.size()) {
      err = "variable " + v.name + " is truncated";
      return false;
    }
    const unsigned char* q = data.data() + v.begin;
    for (uint64_t k = 0; k < count; ++k, q += sz) {
      if (sz == 8) {
        uint64_t u = 0;
        for (int s = 0; s < 8; ++s) u = u << 8 | q[s];
        std::memcpy(&dst[k], &u, 8);
      } else {
        uint32_t u = 0;
        for (int s = 0; s < 4; ++s) u = u << 8 | q[s];
        float x;
        std::memcpy(&x, &u, 4);
        dst[k] = x;
      }
    }
    return true;
  }
};

bool open_file(const std::string& path, File& F, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  unsigned char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0)
    F.data.insert(F.data.end(), chunk, chunk + got);
  std::fclose(f);
  const std::vector<unsigned char>& data = F.data;
  if (data.size() >= 8 && std::memcmp(data.data(), "\x89HDF\r\n\x1a\n", 8) == 0) {
    err = path + " is a NetCDF-4 (HDF5) file; this library reads NetCDF classic and "
                 "64-bit-offset files";
    return false;
  }
  if (data.size() < 4 || std::memcmp(data.data(), "CDF", 3) != 0 || (data[3] != 1 && data[3] != 2)) {
    err = path + " is not a NetCDF classic file";
    return false;
  }
  const bool off64 = data[3] == 2;
  In in{data.data(), data.size()};
  in.o = 4;
  in.u32();  // numrecs
  {
    const uint32_t tag = in.u32(), cnt = in.u32();
    if (!(tag == 0 && cnt == 0)) {
      if (tag != kDimTag) in.ok = false;
      for (uint32_t d = 0; d < cnt && in.ok; ++d) {
        std::string nm = in.name();
        F.dims.emplace_back(nm, in.u32());
      }
    }
  }
  in.skip_atts();
  {
    const uint32_t tag = in.u32(), cnt = in.u32();
    if (!(tag == 0 && cnt == 0)) {
      if (tag != kVarTag) in.ok = false;
      for (uint32_t v = 0; v < cnt && in.ok; ++v) {
        Var var;
        var.name = in.name();
        const uint32_t nd = in.u32();
        for (uint32_t d = 0; d < nd && in.ok; ++d) var.dims.push_back(in.u32());
        in.skip_atts();
        var.type = in.u32();
        in.u32();  // vsize
        var.begin = off64 ? in.u64() : in.u32();
        F.vars.push_back(var);
      }
    }
  }
  if (!in.ok) {
    err = path + ": malformed NetCDF header";
    return false;
  }
  for (const Var& v : F.vars)
    for (uint32_t d : v.dims)
      if (d >= F.dims.size() || F.dims[d].second == 0) {
        err = path + ": record (unlimited) or unknown dimensions are not supported";
        return false;
      }
  return true;
}

std::string mismatch(uint32_t fnx, uint32_t fny, int nx, int ny) {
  return "grid mismatch: file has " + std::to_string(fnx) + " x " + std::to_string(fny) +
         " but the simulation expects " + std::to_string(nx) + " x " + std::to_string(ny);
}

}  // namespace

int read_restart(const std::string& path, int nx, int ny, double* h, double* hu, double* hv,
                 double* b, double& time, std::string& err) {
  File F;
  if (!open_file(path, F, err)) return -1;
  const int fx = F.dim("x"), fy = F.dim("y");
  if (fx < 0 || fy < 0) {
    err = path + ": dimensions x and y not found";
    return -1;
  }
  if ((int)F.dims[fx].second != nx || (int)F.dims[fy].second != ny) {
    err = "restart " + mismatch(F.dims[fx].second, F.dims[fy].second, nx, ny);
    return 1;
  }
  const uint64_t n2 = (uint64_t)nx * (uint64_t)ny;
  auto field = [&](const char* nm, double* dst, uint64_t count) -> bool {
    const Var* v = F.var(nm);
    if (!v) {
      err = path + ": variable " + nm + " not found";
      return false;
    }
    const bool shape_ok = count == 1 ? v->dims.empty()
                                     : (v->dims.size() == 2 && v->dims[0] == (uint32_t)fy &&
                                        v->dims[1] == (uint32_t)fx);
    if (!shape_ok) {
      err = path + ": variable " + nm + " has an unexpected shape";
      return false;
    }
    if (!F.values(*v, count, dst, err)) {
      err = path + ": " + err;
      return false;
    }
    return true;
  };
  if (!field("h", h, n2) || !field("hu", hu, n2) || !field("hv", hv, n2) || !field("b", b, n2) ||
      !field("time", &time, 1))
    return -1;
  return 0;
}

// load_bathymetry_into_array (src/io/rki_bathymetry.F90:21-138): variable b,
// elevation or depth (first found) over dimensions x, y in either order.
int read_bathymetry(const std::string& path, int nx, int ny, double* b, std::string& err) {
  File F;
  if (!open_file(path, F, err)) return -1;
  const int fx = F.dim("x"), fy = F.dim("y");
  if (fx < 0 || fy < 0) {
    err = path + ": dimensions x and y not found";
    return -1;
  }
  const Var* v = nullptr;
  for (const char* nm : {"b", "elevation", "depth"})
    if (!v) v = F.var(nm);
  if (!v) {
    err = path + ": no bathymetry variable (tried: b, elevation, depth)";
    return -1;
  }
  if (v->dims.size() != 2) {
    err = path + ": bathymetry variable " + v->name + " is not 2-D";
    return -1;
  }
  // file (row-major) dims (y, x): x varies fastest, as in the Fortran array;
  // (x, y): a C-order b[x][y], read transposed
  const bool transposed = v->dims[1] == (uint32_t)fy;
  const uint32_t fnx = F.dims[transposed ? v->dims[0] : v->dims[1]].second;
  const uint32_t fny = F.dims[transposed ? v->dims[1] : v->dims[0]].second;
  if ((int)fnx != nx || (int)fny != ny) {
    err = "bathymetry " + mismatch(fnx, fny, nx, ny);
    return 1;
  }
  const uint64_t n2 = (uint64_t)nx * (uint64_t)ny;
  std::vector<double> tmp(n2);
  if (!F.values(*v, n2, tmp.data(), err)) {
    err = path + ": " + err;
    return -1;
  }
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i)
      b[(size_t)i + (size_t)j * nx] =
          transposed ? tmp[(size_t)j + (size_t)i * ny] : tmp[(size_t)i + (size_t)j * nx];
  return 0;
}

}  // namespace nc
}  // namespace rkb
