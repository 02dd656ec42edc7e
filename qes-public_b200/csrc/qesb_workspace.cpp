// Workspace files: the solve's inputs and winds in NetCDF classic format.
//
// The reference writes a "workspace" file per run through netCDF-C++
// (src/winds/WINDSOutputWorkspace.cpp:40-154, over src/util/QESNetCDFOutput.cpp)
// and can re-read its solver coefficients from one
// (src/winds/WINDSGeneralData.cpp:880-910). The library writes the same
// dimensions, variables, layouts and attributes (units, long_name) for the
// fields on the solve's path, in the NetCDF classic format with 64-bit offsets
// (CDF-2), which netCDF-C, and so the reference's NetCDFInput, reads like any
// NetCDF file, and reads classic files (CDF-1 and CDF-2) back, whoever wrote
// them. NetCDF-4 (HDF5) files, the netCDF-C++ default, are refused with a
// message naming the conversion (nccopy -k 2).
//
// Classic format, as Unidata's specification gives it: a big-endian header
// (magic "CDF" + version, record count, dimension list, global attribute
// list, variable list with each variable's dimension ids, attributes, type,
// size and file offset), then the fixed-size variables' data, then the
// records, each holding one slab of every record variable in turn. Names and
// attribute values are padded to 4 bytes.
//
// Written fields (record dimension "t", one record):
//   t(t) double; x_face, y_face, z_face, x, y, z coordinates (float);
//   u, v, w, u0, v0, w0 (t, z_face, y_face, x_face) float;
//   dz_array(z) float; icellflag (t, z, y, x) int; e, f, g, h, m, n (t, z, y, x) float.
// Coordinates follow WINDSOutputWorkspace.cpp:50-88: x, y, z are the cell
// centres (Domain::x, y, z); x_face = {x[0] - dx, x[0], ..., x[nx-2]},
// y_face = {y[0] - dy, y[0] + dy, ..., y[ny-2] + dy}, z_face = Domain::z_face.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "qesb.h"
#include "qesb_internal.h"

#define CKS(expr)                  \
  do {                             \
    const qesb_status s_ = (expr); \
    if (s_ != QESB_OK) return s_;  \
  } while (0)

namespace {

enum NcType { kByte = 1, kChar = 2, kShort = 3, kInt = 4, kFloat = 5, kDouble = 6 };
constexpr uint32_t kTagDim = 0x0A, kTagVar = 0x0B, kTagAtt = 0x0C;

int type_size(int t)
{
  switch (t) {
  case kByte:
  case kChar: return 1;
  case kShort: return 2;
  case kInt:
  case kFloat: return 4;
  case kDouble: return 8;
  default: return 0;
  }
}
size_t pad4(size_t n) { return (n + 3) & ~size_t(3); }

// ---------------------------------------------------------------- writing
struct Out {
  std::vector<unsigned char> b;
  void u32(uint32_t v)
  {
    for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
  }
  void u64(uint64_t v)
  {
    for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
  }
  void name(const std::string &s)
  {
    u32((uint32_t)s.size());
    b.insert(b.end(), s.begin(), s.end());
    while (b.size() % 4) b.push_back(0);
  }
};

struct WVar {
  std::string name, units, long_name;
  std::vector<int> dims;  // dimension ids
  int type;
  const void *data;       // host data in C order of dims
  size_t count;           // elements (one record for record variables)
  bool record;
  size_t vsize = 0;       // bytes per variable (or per record), padded to 4
  size_t begin_pos = 0;   // header position of the 8-byte begin field
};

void put_be(unsigned char *dst, const void *src, size_t n, int tsize)
{
  const unsigned char *s = static_cast<const unsigned char *>(src);
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < tsize; ++k) dst[i * tsize + k] = s[i * tsize + (tsize - 1 - k)];
}

// ---------------------------------------------------------------- reading
struct In {
  const unsigned char *p, *end;
  bool ok = true;
  uint32_t u32()
  {
    if (end - p < 4) return ok = false, 0u;
    const uint32_t v = (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3];
    p += 4;
    return v;
  }
  uint64_t u64()
  {
    const uint64_t hi = u32();
    return hi << 32 | u32();
  }
  std::string name()
  {
    const uint32_t n = u32();
    if (!ok || (size_t)(end - p) < pad4(n)) return ok = false, std::string();
    std::string s(reinterpret_cast<const char *>(p), n);
    p += pad4(n);
    return s;
  }
  void skip(size_t n)
  {
    if ((size_t)(end - p) < n) ok = false;
    else p += n;
  }
};

struct RDim {
  std::string name;
  uint64_t len;
};
struct RVar {
  std::string name;
  std::vector<uint32_t> dims;
  int type;
  uint64_t vsize, begin;
};
struct NcFile {
  std::string path;
  uint64_t size = 0;  // bytes in the file
  uint64_t numrecs = 0, recsize = 0;
  int rec_dim = -1;
  std::vector<RDim> dims;
  std::vector<RVar> vars;
};

qesb_status skip_atts(In &in)
{
  const uint32_t tag = in.u32(), n = in.u32();
  if (tag == 0 && n == 0) return QESB_OK;
  if (tag != kTagAtt) return qesb_fail(QESB_ERR_ARG, "workspace: bad attribute list");
  for (uint32_t a = 0; a < n && in.ok; ++a) {
    in.name();
    const int t = (int)in.u32();
    const uint32_t ne = in.u32();
    if (!type_size(t)) return qesb_fail(QESB_ERR_ARG, "workspace: bad attribute type %d", t);
    in.skip(pad4((size_t)ne * type_size(t)));
  }
  return in.ok ? QESB_OK : qesb_fail(QESB_ERR_ARG, "workspace: truncated header");
}

// Parses the header in bytes [0, n) of a file of `size` bytes; *truncated
// reports a header that runs past n (the caller then reads a longer prefix).
qesb_status nc_parse(const unsigned char *b, size_t n, NcFile &f, bool *truncated)
{
  *truncated = false;
  f.dims.clear();
  f.vars.clear();
  f.rec_dim = -1;
  f.recsize = 0;
  const char *path = f.path.c_str();
  if (n >= 4 && b[0] == 0x89 && b[1] == 'H' && b[2] == 'D' && b[3] == 'F')
    return qesb_fail(QESB_ERR_ARG,
                     "workspace: %s is NetCDF-4 (HDF5); convert it to the classic format first "
                     "(nccopy -k 2 in.nc out.nc)",
                     path);
  if (n < 8 || b[0] != 'C' || b[1] != 'D' || b[2] != 'F' || (b[3] != 1 && b[3] != 2))
    return qesb_fail(QESB_ERR_ARG, "workspace: %s is not a NetCDF classic (CDF-1 / CDF-2) file", path);
  const bool off64 = b[3] == 2;
  In in{b + 4, b + n};
  f.numrecs = in.u32();
  if (f.numrecs == 0xFFFFFFFFu) return qesb_fail(QESB_ERR_ARG, "workspace: streaming record count not supported");
  uint32_t tag = in.u32(), cnt = in.u32();
  if (!(tag == 0 && cnt == 0)) {
    if (tag != kTagDim) return qesb_fail(QESB_ERR_ARG, "workspace: bad dimension list");
    for (uint32_t d = 0; d < cnt && in.ok; ++d) {
      RDim dim;
      dim.name = in.name();
      dim.len = in.u32();
      if (dim.len == 0) f.rec_dim = (int)d;
      f.dims.push_back(dim);
    }
  }
  if (!in.ok) return *truncated = true, QESB_ERR_ARG;
  {
    const qesb_status st = skip_atts(in);
    if (!in.ok) return *truncated = true, QESB_ERR_ARG;
    if (st != QESB_OK) return st;
  }
  tag = in.u32();
  cnt = in.u32();
  if (!(tag == 0 && cnt == 0) && in.ok) {
    if (tag != kTagVar) return qesb_fail(QESB_ERR_ARG, "workspace: bad variable list");
    for (uint32_t v = 0; v < cnt && in.ok; ++v) {
      RVar var;
      var.name = in.name();
      const uint32_t nd = in.u32();
      for (uint32_t d = 0; d < nd && in.ok; ++d) var.dims.push_back(in.u32());
      const qesb_status st = skip_atts(in);
      if (!in.ok) break;
      if (st != QESB_OK) return st;
      var.type = (int)in.u32();
      var.vsize = in.u32();
      var.begin = off64 ? in.u64() : in.u32();
      if (!in.ok) break;
      if (!type_size(var.type)) return qesb_fail(QESB_ERR_ARG, "workspace: bad type of %s", var.name.c_str());
      for (uint32_t d : var.dims)
        if (d >= f.dims.size()) return qesb_fail(QESB_ERR_ARG, "workspace: bad dimension id in %s", var.name.c_str());
      f.vars.push_back(var);
    }
  }
  if (!in.ok) return *truncated = true, QESB_ERR_ARG;

  // record size: the record variables' slabs (one record variable: unpadded)
  int nrec = 0;
  for (const RVar &v : f.vars)
    if (!v.dims.empty() && (int)v.dims[0] == f.rec_dim) {
      ++nrec;
      f.recsize += v.vsize;
    }
  if (nrec == 1)
    for (const RVar &v : f.vars)
      if (!v.dims.empty() && (int)v.dims[0] == f.rec_dim) {
        uint64_t c = type_size(v.type);
        for (size_t d = 1; d < v.dims.size(); ++d) c *= f.dims[v.dims[d]].len;
        f.recsize = c;
      }
  return QESB_OK;
}

// Opens a classic file: its size and header (read as a prefix that grows until
// the header fits); the data stay on disk until read_var.
qesb_status nc_open(const char *path, NcFile &f)
{
  f.path = path;
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return qesb_fail(QESB_ERR_ARG, "workspace: cannot open %s", path);
  std::fseek(fp, 0, SEEK_END);
  const long fsize = std::ftell(fp);
  f.size = fsize > 0 ? (uint64_t)fsize : 0;
  std::vector<unsigned char> buf;
  for (uint64_t cap = 1 << 16;; cap *= 8) {
    const size_t n = (size_t)std::min<uint64_t>(cap, f.size);
    buf.resize(n);
    std::fseek(fp, 0, SEEK_SET);
    if (std::fread(buf.data(), 1, n, fp) != n) {
      std::fclose(fp);
      return qesb_fail(QESB_ERR_ARG, "workspace: cannot read %s", path);
    }
    bool truncated = false;
    const qesb_status st = nc_parse(buf.data(), n, f, &truncated);
    if (st == QESB_OK || !truncated || n == f.size) {
      std::fclose(fp);
      if (truncated) return qesb_fail(QESB_ERR_ARG, "workspace: truncated header in %s", path);
      return st;
    }
  }
}

const RVar *find_var(const NcFile &f, const char *name)
{
  for (const RVar &v : f.vars)
    if (v.name == name) return &v;
  return nullptr;
}
uint64_t dim_len(const NcFile &f, const char *name)
{
  for (const RDim &d : f.dims)
    if (d.name == name) return d.len;
  return 0;
}

// Reads variable `name` (record 0 for record variables) as `want` elements,
// converting to float (kFloat) or int (kInt).
qesb_status read_var(const NcFile &f, const char *name, size_t want, int as, void *out)
{
  const RVar *v = find_var(f, name);
  if (!v) return qesb_fail(QESB_ERR_ARG, "workspace: variable %s missing", name);
  const bool rec = !v->dims.empty() && (int)v->dims[0] == f.rec_dim;
  if (rec && f.numrecs < 1) return qesb_fail(QESB_ERR_ARG, "workspace: %s has no record", name);
  uint64_t count = 1;
  for (size_t d = rec ? 1 : 0; d < v->dims.size(); ++d) count *= f.dims[v->dims[d]].len;
  if (count != want)
    return qesb_fail(QESB_ERR_ARG, "workspace: %s holds %llu values, the grid needs %zu", name,
                     (unsigned long long)count, want);
  const int ts = type_size(v->type);
  if (v->begin + count * ts > f.size) return qesb_fail(QESB_ERR_ARG, "workspace: %s runs past the file", name);
  if (v->type == kChar) return qesb_fail(QESB_ERR_ARG, "workspace: %s has a text type", name);
  FILE *fp = std::fopen(f.path.c_str(), "rb");
  if (!fp) return qesb_fail(QESB_ERR_ARG, "workspace: cannot open %s", f.path.c_str());
  if (fseeko(fp, (off_t)v->begin, SEEK_SET) != 0) {
    std::fclose(fp);
    return qesb_fail(QESB_ERR_ARG, "workspace: cannot seek to %s", name);
  }
  constexpr size_t kChunk = 1 << 20;  // values per read
  std::vector<unsigned char> buf(std::min(want, kChunk) * ts);
  for (size_t i0 = 0; i0 < want; i0 += kChunk) {
    const size_t n = std::min(kChunk, want - i0);
    if (std::fread(buf.data(), 1, n * ts, fp) != n * ts) {
      std::fclose(fp);
      return qesb_fail(QESB_ERR_ARG, "workspace: short read of %s", name);
    }
    for (size_t i = 0; i < n; ++i) {
      const unsigned char *e = buf.data() + i * ts;
      double x = 0.0;
      switch (v->type) {
      case kByte: x = (double)(int8_t)e[0]; break;
      case kShort: x = (double)(int16_t)((uint16_t)e[0] << 8 | e[1]); break;
      case kInt: x = (double)(int32_t)((uint32_t)e[0] << 24 | (uint32_t)e[1] << 16 | (uint32_t)e[2] << 8 | e[3]); break;
      case kFloat: {
        const uint32_t u = (uint32_t)e[0] << 24 | (uint32_t)e[1] << 16 | (uint32_t)e[2] << 8 | e[3];
        float fl;
        std::memcpy(&fl, &u, 4);
        x = fl;
        break;
      }
      default: {
        uint64_t u = 0;
        for (int k = 0; k < 8; ++k) u = u << 8 | e[k];
        std::memcpy(&x, &u, 8);
        break;
      }
      }
      if (as == kFloat) static_cast<float *>(out)[i0 + i] = (float)x;
      else static_cast<int *>(out)[i0 + i] = (int)x;
    }
  }
  std::fclose(fp);
  return QESB_OK;
}

}  // namespace

extern "C" {

qesb_status qesb_workspace_write(const char *path, const qesb_grid *g, double t, const float *u, const float *v,
                                 const float *w, const float *u0, const float *v0, const float *w0,
                                 const int *icellflag, const float *e, const float *f, const float *gc,
                                 const float *h, const float *m, const float *n)
{
  if (!path || !g || !g->dz_array || !u || !v || !w || !u0 || !v0 || !w0 || !icellflag || !e || !f || !gc || !h ||
      !m || !n)
    return qesb_fail(QESB_ERR_ARG, "qesb_workspace_write: null argument");
  if (g->Nx < 1 || g->Ny < 1 || g->Nz < 1) return qesb_fail(QESB_ERR_ARG, "qesb_workspace_write: bad grid");
  const int nx = g->Nx + 1, ny = g->Ny + 1, nz = g->Nz + 2;
  const size_t nf = (size_t)nx * ny * nz, nc = (size_t)(nx - 1) * (ny - 1) * (nz - 1);
  // coordinates (Domain.cpp:121-151 for z; WINDSOutputWorkspace.cpp:50-88)
  std::vector<float> x(nx - 1), y(ny - 1), z(nz - 1), zf(nz), xf(nx), yf(ny), dz(g->dz_array, g->dz_array + nz - 1);
  for (int i = 0; i < nx - 1; ++i) x[i] = (i + 0.5f) * g->dx;
  for (int j = 0; j < ny - 1; ++j) y[j] = (j + 0.5f) * g->dy;
  zf[0] = -dz[0];
  zf[1] = 0.0f;
  for (int k = 2; k < nz; ++k) zf[k] = zf[k - 1] + dz[k - 1];
  z[0] = -0.5f * dz[0];
  for (int k = 1; k < nz - 1; ++k) z[k] = 0.5f * (zf[k] + zf[k + 1]);
  xf[0] = x[0] - g->dx;
  for (int i = 0; i < nx - 1; ++i) xf[i + 1] = x[i];
  yf[0] = y[0] - g->dy;
  for (int j = 0; j < ny - 1; ++j) yf[j + 1] = y[j] + g->dy;

  // dimensions: 0 t (record), 1 x_face, 2 y_face, 3 z_face, 4 x, 5 y, 6 z
  const char *dname[7] = {"t", "x_face", "y_face", "z_face", "x", "y", "z"};
  const uint32_t dlen[7] = {0, (uint32_t)nx, (uint32_t)ny, (uint32_t)nz, (uint32_t)(nx - 1), (uint32_t)(ny - 1),
                            (uint32_t)(nz - 1)};
  std::vector<WVar> vars = {
      {"t", "s", "time since start of simulation", {0}, kDouble, &t, 1, true},
      {"x_face", "m", "x-face", {1}, kFloat, xf.data(), xf.size(), false},
      {"y_face", "m", "y-face", {2}, kFloat, yf.data(), yf.size(), false},
      {"z_face", "m", "z-face", {3}, kFloat, zf.data(), zf.size(), false},
      {"u", "m s-1", "x-component velocity", {0, 3, 2, 1}, kFloat, u, nf, true},
      {"v", "m s-1", "y-component velocity", {0, 3, 2, 1}, kFloat, v, nf, true},
      {"w", "m s-1", "z-component velocity", {0, 3, 2, 1}, kFloat, w, nf, true},
      {"u0", "m s-1", "x-component initial velocity", {0, 3, 2, 1}, kFloat, u0, nf, true},
      {"v0", "m s-1", "y-component initial velocity", {0, 3, 2, 1}, kFloat, v0, nf, true},
      {"w0", "m s-1", "z-component initial velocity", {0, 3, 2, 1}, kFloat, w0, nf, true},
      {"x", "m", "x-distance", {4}, kFloat, x.data(), x.size(), false},
      {"y", "m", "y-distance", {5}, kFloat, y.data(), y.size(), false},
      {"z", "m", "z-distance", {6}, kFloat, z.data(), z.size(), false},
      {"dz_array", "m", "dz size of the cells", {6}, kFloat, dz.data(), dz.size(), false},
      {"icellflag", "--", "icell flag value", {0, 6, 5, 4}, kInt, icellflag, nc, true},
      {"e", "--", "e cut-cell coefficient", {0, 6, 5, 4}, kFloat, e, nc, true},
      {"f", "--", "f cut-cell coefficient", {0, 6, 5, 4}, kFloat, f, nc, true},
      {"g", "--", "g cut-cell coefficient", {0, 6, 5, 4}, kFloat, gc, nc, true},
      {"h", "--", "h cut-cell coefficient", {0, 6, 5, 4}, kFloat, h, nc, true},
      {"m", "--", "m cut-cell coefficient", {0, 6, 5, 4}, kFloat, m, nc, true},
      {"n", "--", "n cut-cell coefficient", {0, 6, 5, 4}, kFloat, n, nc, true},
  };
  int nrec = 0;
  for (WVar &wv : vars) {
    wv.vsize = pad4(wv.count * type_size(wv.type));
    nrec += wv.record;
  }
  if (nrec == 1)
    for (WVar &wv : vars)
      if (wv.record) wv.vsize = wv.count * type_size(wv.type);
  for (const WVar &wv : vars)
    if (wv.vsize > 0xFFFFFFFCu) return qesb_fail(QESB_ERR_ARG, "qesb_workspace_write: %s exceeds 4 GB", wv.name.c_str());

  Out o;
  o.b.insert(o.b.end(), {'C', 'D', 'F', 2});
  o.u32(1);  // one record
  o.u32(kTagDim);
  o.u32(7);
  for (int d = 0; d < 7; ++d) {
    o.name(dname[d]);
    o.u32(dlen[d]);
  }
  o.u32(0);  // no global attributes
  o.u32(0);
  o.u32(kTagVar);
  o.u32((uint32_t)vars.size());
  for (WVar &wv : vars) {
    o.name(wv.name);
    o.u32((uint32_t)wv.dims.size());
    for (int d : wv.dims) o.u32((uint32_t)d);
    o.u32(kTagAtt);
    o.u32(2);
    for (int a = 0; a < 2; ++a) {
      const std::string &val = a == 0 ? wv.units : wv.long_name;
      o.name(a == 0 ? "units" : "long_name");
      o.u32(kChar);
      o.name(val);  // count + chars + padding, the layout of a char attribute
    }
    o.u32((uint32_t)wv.type);
    o.u32((uint32_t)wv.vsize);
    wv.begin_pos = o.b.size();
    o.u64(0);  // patched below
  }
  // data: fixed-size variables, then the one record
  uint64_t pos = o.b.size();
  for (int pass = 0; pass < 2; ++pass)
    for (WVar &wv : vars)
      if (wv.record == (pass == 1)) {
        for (int k = 0; k < 8; ++k) o.b[wv.begin_pos + k] = (unsigned char)(pos >> (56 - 8 * k));
        pos += wv.vsize;
      }
  FILE *fp = std::fopen(path, "wb");
  if (!fp) return qesb_fail(QESB_ERR_ARG, "qesb_workspace_write: cannot create %s", path);
  bool good = std::fwrite(o.b.data(), 1, o.b.size(), fp) == o.b.size();
  // each variable in big-endian chunks, then its padding to vsize
  constexpr size_t kChunk = 1 << 20;  // values per write
  std::vector<unsigned char> buf;
  for (int pass = 0; pass < 2 && good; ++pass)
    for (const WVar &wv : vars) {
      if (wv.record != (pass == 1) || !good) continue;
      const int ts = type_size(wv.type);
      const unsigned char *src = static_cast<const unsigned char *>(wv.data);
      for (size_t i0 = 0; i0 < wv.count && good; i0 += kChunk) {
        const size_t n = std::min(kChunk, wv.count - i0);
        buf.resize(n * ts);
        put_be(buf.data(), src + i0 * ts, n, ts);
        good = std::fwrite(buf.data(), 1, n * ts, fp) == n * ts;
      }
      const size_t padn = wv.vsize - wv.count * ts;
      const unsigned char zeros[4] = {0, 0, 0, 0};
      if (good && padn) good = std::fwrite(zeros, 1, padn, fp) == padn;
    }
  const int cl = std::fclose(fp);
  if (!good || cl != 0) return qesb_fail(QESB_ERR_ARG, "qesb_workspace_write: write to %s failed", path);
  return QESB_OK;
}

qesb_status qesb_workspace_dims(const char *path, int *Nx, int *Ny, int *Nz, float *dx, float *dy)
{
  if (!path || !Nx || !Ny || !Nz) return qesb_fail(QESB_ERR_ARG, "qesb_workspace_dims: null argument");
  NcFile f;
  CKS(nc_open(path, f));
  const uint64_t lx = dim_len(f, "x"), ly = dim_len(f, "y"), lz = dim_len(f, "z");
  if (lx < 1 || ly < 1 || lz < 2) return qesb_fail(QESB_ERR_ARG, "workspace: dimensions x, y, z missing");
  *Nx = (int)lx;
  *Ny = (int)ly;
  *Nz = (int)lz - 1;
  std::vector<float> xs(lx), ys(ly);
  if (dx) {
    CKS(read_var(f, "x", lx, kFloat, xs.data()));
    *dx = lx > 1 ? xs[1] - xs[0] : 2.0f * xs[0];
  }
  if (dy) {
    CKS(read_var(f, "y", ly, kFloat, ys.data()));
    *dy = ly > 1 ? ys[1] - ys[0] : 2.0f * ys[0];
  }
  return QESB_OK;
}

qesb_status qesb_workspace_read(const char *path, int Nx, int Ny, int Nz, float *dz_array, int *icellflag,
                                float *e, float *f, float *g, float *h, float *m, float *n, float *u0, float *v0,
                                float *w0, float *u, float *v, float *w)
{
  if (!path) return qesb_fail(QESB_ERR_ARG, "qesb_workspace_read: null path");
  NcFile file;
  CKS(nc_open(path, file));
  if (dim_len(file, "x") != (uint64_t)Nx || dim_len(file, "y") != (uint64_t)Ny ||
      dim_len(file, "z") != (uint64_t)Nz + 1)
    return qesb_fail(QESB_ERR_ARG, "qesb_workspace_read: %s is not a %dx%dx%d grid", path, Nx, Ny, Nz);
  const size_t nc = (size_t)Nx * Ny * (Nz + 1), nf = (size_t)(Nx + 1) * (Ny + 1) * (Nz + 2);
  if (dz_array) CKS(read_var(file, "dz_array", Nz + 1, kFloat, dz_array));
  if (icellflag) CKS(read_var(file, "icellflag", nc, kInt, icellflag));
  const char *cn[6] = {"e", "f", "g", "h", "m", "n"};
  float *cv[6] = {e, f, g, h, m, n};
  for (int q = 0; q < 6; ++q)
    if (cv[q]) CKS(read_var(file, cn[q], nc, kFloat, cv[q]));
  const char *fn[6] = {"u0", "v0", "w0", "u", "v", "w"};
  float *fv[6] = {u0, v0, w0, u, v, w};
  for (int q = 0; q < 6; ++q)
    if (fv[q]) CKS(read_var(file, fn[q], nf, kFloat, fv[q]));
  return QESB_OK;
}

}  // extern "C"
