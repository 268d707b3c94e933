// Superdroplet output: a Zarr v2 dataset with the files CLEO's SuperdropsObserver and
// TimeObserver write into a SimpleDataset<FSStore> (observers/superdrops_observer.hpp:485-490,
// observers/time_observer.hpp:46-144, zarr/simple_dataset.hpp:44-292).
//
// Per array (ZarrArray, zarr/zarr_array.hpp:82-346): a host buffer of `maxchunk` elements whose
// unfilled part holds the type's maximum (zarr/buffer.hpp:57-66). A write fills the buffer;
// a buffer that is full is stored as the next chunk file "<name>/<chunk number>" (chunk_label of
// a 1-D array, zarr/chunks.hpp:88-106) before whole chunks are stored straight from the data and
// the remainder goes to the buffer (zarr_array.hpp:146-162, 313-327). When the dataset is
// closed, a partly filled buffer is stored whole, padding included (zarr_array.hpp:207-216), and
// .zarray gets the final shape: the number of observations for "time" and "raggedcount", the
// number of elements written for a ragged array (xarray_zarr_array.hpp:91-98, 139-143).
// Metadata strings: .zarray (zarr/zarr_metadata.cpp:32-81), .zattrs (zarr/xarray_metadata.cpp:
// 35-170, scale factors in scientific notation with 6 digits), the group's .zgroup and .zattrs
// (zarr/zarr_group.hpp:49-53, zarr/simple_dataset.hpp:68-73). These are file formats and must
// match the reference byte for byte, so the strings follow the reference's exactly.
//
// An observation gathers the domain superdroplets on the GPU (cleo_b200_gather_supers) into
// pinned host staging, then the arrays are written by one host thread each.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <cfloat>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cleo_b200.h"

namespace {

constexpr double kTIME0 = 1000.0;                       // cleoconstants.hpp:74
constexpr double kCOORD0 = kTIME0 * 1.0;                // cleoconstants.hpp:75
constexpr double kR0 = 1e-6;                            // cleoconstants.hpp:80
constexpr double kRHO0 = 100000.0 / (1004.64 * 273.15); // cleoconstants.hpp:83
constexpr double kMASS0grams = kR0 * kR0 * kR0 * kRHO0 * 1000;

bool make_dirs(const std::string& path) {
  std::string cur;
  size_t pos = 0;
  while (pos != std::string::npos) {
    pos = path.find('/', pos + 1);
    cur = path.substr(0, pos);
    if (cur.empty()) continue;
    if (mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return false;
  }
  return true;
}

bool write_file(const std::string& path, const void* data, size_t bytes) {
  int fd = open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (fd < 0) return false;
  const char* p = static_cast<const char*>(data);
  size_t left = bytes;
  while (left > 0) {
    const ssize_t w = write(fd, p, left);
    if (w < 0) {
      if (errno == EINTR) continue;
      close(fd);
      return false;
    }
    p += w;
    left -= (size_t)w;
  }
  return close(fd) == 0;
}

bool write_text(const std::string& path, const std::string& s) {
  return write_file(path, s.data(), s.size());
}

std::string zarray_json(size_t shape, size_t chunk, const char* dtype) {
  return "{\n  \"shape\": [" + std::to_string(shape) + "],\n  \"chunks\": [" +
         std::to_string(chunk) + "],\n  \"dtype\": \"" + dtype +
         "\",\n  \"order\": \"C\",\n  \"compressor\": null,\n  \"fill_value\": null,\n"
         "  \"filters\": null,\n  \"zarr_format\": 2\n}";
}

std::string scale_string(double v) {  // std::scientific, precision 6
  char b[64];
  std::snprintf(b, sizeof b, "%.6e", v);
  return b;
}

// .zattrs of an array: integers carry no scale factor; ragged arrays name their sample dimension
std::string zattrs_json(const char* dim, const char* units, bool floating, double scale,
                        const char* sampledim) {
  std::string s = std::string("{\n  \"_ARRAY_DIMENSIONS\": [\"") + dim + "\"],\n  \"units\": \"" +
                  units + "\"";
  if (floating) s += ",\n  \"scale_factor\": " + scale_string(scale);
  if (sampledim) s += ",\n  \"sample_dimension\": \"" + std::string(sampledim) + "\"";
  return s + "\n}";
}

struct Array1D {
  std::string dir;  // <dataset>/<name>
  const char* dtype;
  size_t esize, chunk;
  std::vector<uint8_t> pad;  // one element of the type's maximum
  std::vector<uint8_t> buf;
  size_t fill = 0, nchunks = 0, shape_written = 0, chunks_at_shape = 0;
  bool ok = true;

  Array1D(const std::string& root, const char* name, const char* dt, size_t es, size_t ch,
          const void* maxval, const std::string& zattrs)
      : dir(root + "/" + name), dtype(dt), esize(es), chunk(ch), pad(es), buf(es * ch) {
    std::memcpy(pad.data(), maxval, es);
    reset();
    ok = make_dirs(dir) && write_text(dir + "/.zarray", zarray_json(0, chunk, dtype)) &&
         write_text(dir + "/.zattrs", zattrs);
  }
  void reset() {
    for (size_t k = 0; k < chunk; ++k) std::memcpy(buf.data() + k * esize, pad.data(), esize);
    fill = 0;
  }
  void store(const void* data) {
    ok = ok && write_file(dir + "/" + std::to_string(nchunks), data, chunk * esize);
    ++nchunks;
  }
  // write_to_array of n elements (ragged arrays)
  void append(const void* data, size_t n) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    const size_t k = n < chunk - fill ? n : chunk - fill;
    if (k) std::memcpy(buf.data() + fill * esize, p, k * esize);
    fill += k;
    p += k * esize;
    size_t rest = n - k;
    if (fill == chunk) {
      store(buf.data());
      reset();
    }
    while (rest >= chunk) {
      store(p);
      p += chunk * esize;
      rest -= chunk;
    }
    if (rest) {  // only after the buffer was stored and reset
      std::memcpy(buf.data(), p, rest * esize);
      fill = rest;
    }
  }
  // write_to_array of one element (time, raggedcount)
  void append_one(const void* elem) {
    if (fill == chunk) {
      store(buf.data());
      reset();
    }
    std::memcpy(buf.data() + fill * esize, elem, esize);
    ++fill;
  }
  size_t total() const { return nchunks * chunk + fill; }
  // the shape is rewritten whenever new chunks were stored since the last rewrite (as the
  // reference's write_arrayshape does), so a reader sees every stored chunk
  void update_shape(size_t shape) {
    if (nchunks != chunks_at_shape && shape != shape_written) {
      ok = ok && write_text(dir + "/.zarray", zarray_json(shape, chunk, dtype));
      shape_written = shape;
      chunks_at_shape = nchunks;
    }
  }
  void finish(size_t shape) {
    ok = ok && write_text(dir + "/.zarray", zarray_json(shape, chunk, dtype));
    if (fill > 0) store(buf.data());
  }
};

struct VarDesc {
  uint32_t bit;
  const char* name;
  const char* dtype;
  size_t esize;
  const char* units;
  bool floating;
  double scale;
};
const VarDesc kVars[8] = {
    {CLEO_OBS_SDID, "sdId", "<u4", 4, "", false, 1.0},
    {CLEO_OBS_SDGBXINDEX, "sdgbxindex", "<u4", 4, "", false, 1.0},
    {CLEO_OBS_XI, "xi", "<u8", 8, "", false, 1.0},
    {CLEO_OBS_RADIUS, "radius", "<f4", 4, "micro-m", true, kR0 * 1e6},
    {CLEO_OBS_MSOL, "msol", "<f4", 4, "g", true, kMASS0grams},
    {CLEO_OBS_COORD3, "coord3", "<f4", 4, "m", true, kCOORD0},
    {CLEO_OBS_COORD1, "coord1", "<f4", 4, "m", true, kCOORD0},
    {CLEO_OBS_COORD2, "coord2", "<f4", 4, "m", true, kCOORD0},
};

const void* member(const cleo_b200_obs_supers* s, uint32_t bit) {
  switch (bit) {
    case CLEO_OBS_SDID: return s->sdid;
    case CLEO_OBS_SDGBXINDEX: return s->sdgbxindex;
    case CLEO_OBS_XI: return s->xi;
    case CLEO_OBS_RADIUS: return s->radius;
    case CLEO_OBS_MSOL: return s->msol;
    case CLEO_OBS_COORD3: return s->coord3;
    case CLEO_OBS_COORD1: return s->coord1;
    default: return s->coord2;
  }
}

}  // namespace

struct cleo_b200_zarr {
  std::string root;
  size_t maxchunk;
  uint32_t interval, vars;
  size_t ntimes = 0;
  std::unique_ptr<Array1D> time, count;
  std::vector<std::pair<uint32_t, std::unique_ptr<Array1D>>> arrays;
  // pinned staging for gathers from a context
  void* pinned = nullptr;
  size_t pinned_cap = 0;
  cleo_b200_obs_supers stage{};

  bool ok() const {
    bool r = time->ok && count->ok;
    for (auto& a : arrays) r = r && a.second->ok;
    return r;
  }
  ~cleo_b200_zarr() {
    if (pinned) cudaFreeHost(pinned);
  }
};

extern "C" {

int cleo_b200_zarr_open(const char* dir, size_t maxchunk, uint32_t interval, uint32_t vars,
                        cleo_b200_zarr** out) {
  if (!dir || !*dir || !out || maxchunk == 0 || interval == 0 || (vars & ~(uint32_t)CLEO_OBS_ALL))
    return CLEO_ERR_ARGUMENT;
  auto z = std::make_unique<cleo_b200_zarr>();
  z->root = dir;
  while (z->root.size() > 1 && z->root.back() == '/') z->root.pop_back();
  z->maxchunk = maxchunk;
  z->interval = interval;
  z->vars = vars;
  if (!make_dirs(z->root) ||
      !write_text(z->root + "/.zgroup", "{\n  \"zarr_format\": 2\n}") ||
      !write_text(z->root + "/.zattrs",
                  "{\n  \"creator\": \"Clara Bayley\",\n  \"title\": \"Dataset from CLEO is "
                  "Xarray and NetCDF compatible Zarr Group of Arrays\"\n}"))
    return CLEO_ERR_IO;
  const float fmax = FLT_MAX;
  const uint32_t umax = std::numeric_limits<uint32_t>::max();
  const uint64_t lmax = std::numeric_limits<uint64_t>::max();
  z->time = std::make_unique<Array1D>(z->root, "time", "<f4", 4, maxchunk, &fmax,
                                      zattrs_json("time", "s", true, kTIME0, nullptr));
  for (const VarDesc& v : kVars) {
    if (!(vars & v.bit)) continue;
    const void* mx = v.esize == 8 ? (const void*)&lmax : v.floating ? (const void*)&fmax
                                                                    : (const void*)&umax;
    z->arrays.emplace_back(
        v.bit, std::make_unique<Array1D>(
                   z->root, v.name, v.dtype, v.esize, maxchunk, mx,
                   zattrs_json("superdroplets", v.units, v.floating, v.scale, "superdroplets")));
  }
  z->count = std::make_unique<Array1D>(z->root, "raggedcount", "<u4", 4, maxchunk, &umax,
                                       zattrs_json("time", "", false, 1.0, "superdroplets"));
  if (!z->ok()) return CLEO_ERR_IO;
  *out = z.release();
  return CLEO_OK;
}

int cleo_b200_zarr_observe_host(cleo_b200_zarr* z, uint32_t t_mdl, const cleo_b200_obs_supers* s,
                                size_t n) {
  if (!z) return CLEO_ERR_ARGUMENT;
  if (t_mdl % z->interval != 0) return CLEO_OK;  // ConstTstepObserver::on_step
  if (n > std::numeric_limits<uint32_t>::max()) return CLEO_ERR_ARGUMENT;
  if (n && !s) return CLEO_ERR_ARGUMENT;
  for (auto& a : z->arrays)
    if (n && !member(s, a.first)) return CLEO_ERR_ARGUMENT;
  if (n && (z->vars & CLEO_OBS_XI)) {  // XiFunc (superdrops_observer.hpp:229-234)
    for (size_t k = 0; k < n; ++k)
      if (s->xi[k] == std::numeric_limits<uint64_t>::max()) return CLEO_ERR_XI_OUTPUT;
  }
  // TimeObserver first (it sets the time dimension that raggedcount's shape follows)
  ++z->ntimes;
  const float t = (float)((double)t_mdl / 100000.0);
  z->time->append_one(&t);
  z->time->update_shape(z->ntimes);
  // the ragged arrays, one thread each when there is enough to write
  const size_t bytes = n * 4;
  if (z->arrays.size() > 1 && bytes >= (size_t(1) << 22)) {
    std::vector<std::thread> th;
    for (auto& a : z->arrays) {
      Array1D* arr = a.second.get();
      const void* src = member(s, a.first);
      th.emplace_back([arr, src, n] {
        arr->append(src, n);
        arr->update_shape(arr->total());
      });
    }
    for (auto& x : th) x.join();
  } else {
    for (auto& a : z->arrays) {
      a.second->append(member(s, a.first), n);
      a.second->update_shape(a.second->total());
    }
  }
  const uint32_t cnt = (uint32_t)n;
  z->count->append_one(&cnt);
  z->count->update_shape(z->ntimes);
  return z->ok() ? CLEO_OK : CLEO_ERR_IO;
}

int cleo_b200_zarr_observe(cleo_b200_zarr* z, cleo_b200_ctx* ctx, uint32_t t_mdl) {
  if (!z || !ctx) return CLEO_ERR_ARGUMENT;
  if (t_mdl % z->interval != 0) return CLEO_OK;
  size_t n = 0;
  int rc = cleo_b200_gather_supers(ctx, z->vars, &z->stage, z->pinned_cap, &n);
  if (rc == CLEO_ERR_CAPACITY) {  // grow the pinned staging to this context's domain size
    if (z->pinned) cudaFreeHost(z->pinned);
    z->pinned = nullptr;
    z->pinned_cap = 0;
    const size_t cap = n + n / 8 + 1024;
    if (cudaHostAlloc(&z->pinned, cap * 36 + 8 * 16, cudaHostAllocDefault) != cudaSuccess) {
      z->pinned = nullptr;
      return CLEO_ERR_CUDA;
    }
    z->pinned_cap = cap;
    uint8_t* p = static_cast<uint8_t*>(z->pinned);
    const size_t a4 = (cap * 4 + 15) / 16 * 16, a8 = (cap * 8 + 15) / 16 * 16;
    z->stage = cleo_b200_obs_supers{};
    z->stage.xi = reinterpret_cast<uint64_t*>(p), p += a8;
    z->stage.sdid = reinterpret_cast<uint32_t*>(p), p += a4;
    z->stage.sdgbxindex = reinterpret_cast<uint32_t*>(p), p += a4;
    z->stage.radius = reinterpret_cast<float*>(p), p += a4;
    z->stage.msol = reinterpret_cast<float*>(p), p += a4;
    z->stage.coord3 = reinterpret_cast<float*>(p), p += a4;
    z->stage.coord1 = reinterpret_cast<float*>(p), p += a4;
    z->stage.coord2 = reinterpret_cast<float*>(p);
    rc = cleo_b200_gather_supers(ctx, z->vars, &z->stage, z->pinned_cap, &n);
  }
  if (rc != CLEO_OK) return rc;
  return cleo_b200_zarr_observe_host(z, t_mdl, &z->stage, n);
}

int cleo_b200_zarr_close(cleo_b200_zarr* z) {
  if (!z) return CLEO_ERR_ARGUMENT;
  z->time->finish(z->ntimes);
  for (auto& a : z->arrays) a.second->finish(a.second->total());
  z->count->finish(z->ntimes);
  const bool ok = z->ok();
  delete z;
  return ok ? CLEO_OK : CLEO_ERR_IO;
}

}  // extern "C"
