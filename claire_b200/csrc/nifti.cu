// NIfTI-1 file input / output and the image preparation of the file path.
//
// Reference: ReadWriteReg::ReadNII / WriteNII / AllocateImage
// (src/ReadWriteReg.cpp:794-1128, 1130-1475) over nifticlib 2.0.0, which is
// not part of the reference tree; the single-file NIfTI-1 format (348-byte
// header, optional 4-byte extension flag, voxels at vox_offset, x fastest) is
// restated here from its published specification, with zlib for .nii.gz.
// CLAIRE maps the file's (nx, ny, nz) to its grid as nx[0] = nz, nx[1] = ny,
// nx[2] = nx (src/ReadWriteReg.cpp:813-815), so with x3 fastest in memory the
// voxel array is used in file order; values are cast to float without the
// header's scl_slope / scl_inter, as ReadNII does (:1099-1115).
//
// Preparation of read images: CLAIREInterface::SetReferenceImage /
// SetTemplateImage normalise intensities (Normalize, src/CLAIREUtils.cpp:492-525)
// and SetupData smooths them (Preprocessing::Smooth, src/CLAIREInterface.cpp:594-626);
// claire_b200_preprocess does both on the device.
#include <zlib.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/claire_b200.h"
#include "reduce.cuh"
#include "sl.cuh"
#include "spectral.cuh"

namespace {

constexpr int kHdr = 348;

template <typename T>
T get(const unsigned char* h, int off, bool swap) {
  T v;
  std::memcpy(&v, h + off, sizeof(T));
  if (swap) {
    unsigned char b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));
    std::reverse(b, b + sizeof(T));
    std::memcpy(&v, b, sizeof(T));
  }
  return v;
}

template <typename T>
void put(unsigned char* h, int off, T v) {
  std::memcpy(h + off, &v, sizeof(T));
}

int type_bytes(int datatype) {
  switch (datatype) {
    case 2: case 256: return 1;        // uint8, int8
    case 4: case 512: return 2;        // int16, uint16
    case 8: case 768: case 16: return 4;  // int32, uint32, float32
    case 64: case 1024: case 1280: return 8;  // float64, int64, uint64
    default: return 0;
  }
}

template <typename T>
void convert(const unsigned char* src, float* dst, long long n, bool swap) {
  for (long long i = 0; i < n; ++i) {
    T v;
    std::memcpy(&v, src + i * sizeof(T), sizeof(T));
    if (swap && sizeof(T) > 1) {
      unsigned char b[sizeof(T)];
      std::memcpy(b, &v, sizeof(T));
      std::reverse(b, b + sizeof(T));
      std::memcpy(&v, b, sizeof(T));
    }
    dst[i] = static_cast<float>(v);
  }
}

bool ends_with(const std::string& s, const char* suf) {
  const size_t k = std::strlen(suf);
  return s.size() >= k && s.compare(s.size() - k, k, suf) == 0;
}

struct Gz {
  gzFile f = nullptr;
  ~Gz() {
    if (f) gzclose(f);
  }
};

bool read_exact(gzFile f, void* dst, long long bytes) {
  unsigned char* p = static_cast<unsigned char*>(dst);
  while (bytes > 0) {
    const unsigned chunk = (unsigned)std::min<long long>(bytes, 1 << 30);
    const int got = gzread(f, p, chunk);
    if (got <= 0) return false;
    p += got;
    bytes -= got;
  }
  return true;
}

// Min / max normalisation of one scalar field in place (Normalize, nc == 1):
// negative values are set to zero first (and the shift is then 0); then
// x <- (x - xmin) / xmax, with xmax the maximum of the input, as the
// reference computes it.  k_minmax folds the field-statistics partials into
// {xmin, 1 / xmax}.
__global__ void k_minmax(double* parts, int np) {
  double mn = INFINITY, mx = -INFINITY;
  for (int i = threadIdx.x; i < np; i += 32) {
    mn = fmin(mn, parts[np + i]);
    mx = fmax(mx, parts[2 * np + i]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if (threadIdx.x == 0) {
    parts[3 * np] = mn < 0.0 ? 0.0 : mn;
    parts[3 * np + 1] = 1.0 / mx;
  }
}

__global__ void k_normalize(float* x, long long n, const double* __restrict__ mm) {
  const float xmin = (float)mm[0], inv = (float)mm[1];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float v = x[i] < 0.f ? 0.f : x[i];
    x[i] = (v - xmin) * inv;
  }
}

}  // namespace

extern "C" {

int claire_b200_read_nifti(const char* path, int nx[3], float* data, long long capacity) {
  if (!path || !nx) return CB_ERR_ARG;
  // two-file NIfTI-1 (.hdr + .img, either name given, optionally .gz)
  std::string hdr_path(path), img_path;
  for (const char* gz : {"", ".gz"}) {
    const std::string hs = std::string(".hdr") + gz, is = std::string(".img") + gz;
    if (ends_with(hdr_path, hs.c_str())) img_path = hdr_path.substr(0, hdr_path.size() - hs.size()) + is;
    else if (ends_with(hdr_path, is.c_str())) {
      img_path = hdr_path;
      hdr_path = hdr_path.substr(0, hdr_path.size() - is.size()) + hs;
    }
  }
  Gz gz;
  gz.f = gzopen(hdr_path.c_str(), "rb");
  if (!gz.f) return CB_ERR_ARG;
  unsigned char h[kHdr];
  if (!read_exact(gz.f, h, kHdr)) return CB_ERR_ARG;
  bool swap = false;
  int hs = get<int>(h, 0, false);
  if (hs != kHdr) {
    swap = true;
    hs = get<int>(h, 0, true);
    if (hs != kHdr) return CB_ERR_ARG;  // not a NIfTI-1 header
  }
  const bool pair = std::memcmp(h + 344, "ni1", 4) == 0;
  if (!pair && std::memcmp(h + 344, "n+1", 4) != 0) return CB_ERR_ARG;  // not NIfTI-1
  if (pair && img_path.empty()) return CB_ERR_ARG;  // a pair header needs a .hdr / .img name
  const int ndim = get<short>(h, 40, swap);
  long long dim[8];
  for (int i = 0; i < 8; ++i) dim[i] = get<short>(h, 40 + 2 * i, swap);
  if (ndim < 3 || ndim > 7 || dim[1] < 1 || dim[2] < 1 || dim[3] < 1) return CB_ERR_ARG;
  for (int i = 4; i <= ndim; ++i)
    if (dim[i] > 1) return CB_ERR_UNSUPPORTED;  // one scalar volume (one time point, one component)
  const int datatype = get<short>(h, 70, swap);
  const int tb = type_bytes(datatype);
  if (!tb) return CB_ERR_UNSUPPORTED;
  nx[0] = (int)dim[3];
  nx[1] = (int)dim[2];
  nx[2] = (int)dim[1];
  const long long n = dim[1] * dim[2] * dim[3];
  if (!data) return CB_OK;
  if (capacity < n) return CB_ERR_TOO_LARGE;
  const long long off = (long long)get<float>(h, 108, swap);
  // single file: voxels at vox_offset (>= 348) of the same file; pair: at
  // vox_offset (usually 0) of the .img file
  Gz img;
  gzFile src = gz.f;
  long long skip_bytes = off - kHdr;
  if (pair) {
    img.f = gzopen(img_path.c_str(), "rb");
    if (!img.f) return CB_ERR_ARG;
    src = img.f;
    skip_bytes = off;
  }
  if (skip_bytes < 0) return CB_ERR_ARG;
  std::vector<unsigned char> skip((size_t)skip_bytes);
  if (!skip.empty() && !read_exact(src, skip.data(), (long long)skip.size())) return CB_ERR_ARG;
  std::vector<unsigned char> raw((size_t)(n * tb));
  if (!read_exact(src, raw.data(), n * tb)) return CB_ERR_ARG;
  switch (datatype) {
    case 2: convert<uint8_t>(raw.data(), data, n, swap); break;
    case 256: convert<int8_t>(raw.data(), data, n, swap); break;
    case 4: convert<int16_t>(raw.data(), data, n, swap); break;
    case 512: convert<uint16_t>(raw.data(), data, n, swap); break;
    case 8: convert<int32_t>(raw.data(), data, n, swap); break;
    case 768: convert<uint32_t>(raw.data(), data, n, swap); break;
    case 16: convert<float>(raw.data(), data, n, swap); break;
    case 64: convert<double>(raw.data(), data, n, swap); break;
    case 1024: convert<int64_t>(raw.data(), data, n, swap); break;
    case 1280: convert<uint64_t>(raw.data(), data, n, swap); break;
    default: return CB_ERR_UNSUPPORTED;
  }
  return CB_OK;
}

int claire_b200_write_nifti(const char* path, const int nx[3], const float* data) {
  if (!path || !nx || !data || nx[0] < 1 || nx[1] < 1 || nx[2] < 1) return CB_ERR_ARG;
  if (nx[0] > 32767 || nx[1] > 32767 || nx[2] > 32767) return CB_ERR_TOO_LARGE;
  unsigned char h[kHdr + 4];
  std::memset(h, 0, sizeof(h));
  put<int>(h, 0, kHdr);
  // dim: 5 dimensions, (nx, ny, nz) = (nx[2], nx[1], nx[0]), one time point,
  // one component (AllocateImage, src/ReadWriteReg.cpp:1379-1475)
  const short dim[8] = {5, (short)nx[2], (short)nx[1], (short)nx[0], 1, 1, 1, 1};
  for (int i = 0; i < 8; ++i) put<short>(h, 40 + 2 * i, dim[i]);
  put<short>(h, 70, 16);  // float32
  put<short>(h, 72, 32);  // bitpix
  const float pixdim[8] = {1.f, (float)(2.0 * 3.14159265358979323846 / nx[0]),
                           (float)(2.0 * 3.14159265358979323846 / nx[1]),
                           (float)(2.0 * 3.14159265358979323846 / nx[2]), 1.f, 1.f, 1.f, 1.f};
  for (int i = 0; i < 8; ++i) put<float>(h, 76 + 4 * i, pixdim[i]);
  const std::string p(path);
  const bool gzip = ends_with(p, ".gz");
  // .hdr / .img (optionally .gz): the NIfTI-1 pair (NIFTI_FTYPE_NIFTI1_2,
  // src/ReadWriteReg.cpp:1305-1306), header with magic "ni1" and the voxels
  // at offset 0 of the .img file
  std::string base;
  for (const char* suf : {".hdr", ".img", ".hdr.gz", ".img.gz"})
    if (ends_with(p, suf)) base = p.substr(0, p.size() - std::strlen(suf));
  const bool pair = !base.empty();
  put<float>(h, 108, pair ? 0.f : 352.f);  // vox_offset
  put<float>(h, 112, 1.f);                 // scl_slope
  std::memcpy(h + 344, pair ? "ni1" : "n+1", 4);
  const long long n = (long long)nx[0] * nx[1] * nx[2];
  const char* mode = gzip ? "wb6" : "wbT";  // "T": plain (uncompressed) output
  gzFile f = nullptr;
  bool ok = true;
  if (pair) {
    gzFile fh = gzopen((base + (gzip ? ".hdr.gz" : ".hdr")).c_str(), mode);
    if (!fh) return CB_ERR_ARG;
    ok = gzwrite(fh, h, sizeof(h)) == (int)sizeof(h);
    ok = (gzclose(fh) == Z_OK) && ok;
    f = gzopen((base + (gzip ? ".img.gz" : ".img")).c_str(), mode);
  } else {
    f = gzopen(path, mode);
    if (f) ok = gzwrite(f, h, sizeof(h)) == (int)sizeof(h);
  }
  if (!f) return CB_ERR_ARG;
  const unsigned char* src = reinterpret_cast<const unsigned char*>(data);
  long long left = n * 4;
  while (ok && left > 0) {
    const unsigned chunk = (unsigned)std::min<long long>(left, 1 << 30);
    ok = gzwrite(f, src, chunk) == (int)chunk;
    src += chunk;
    left -= chunk;
  }
  ok = (gzclose(f) == Z_OK) && ok;
  return ok ? CB_OK : CB_ERR_ARG;
}

// ReadBIN / WriteBIN (src/ReadWriteReg.cpp:1476-1535): a PETSc binary vector
// (VecLoad / VecView): big-endian int32 class id 1211214, int32 length, then
// the values big-endian, 8 bytes each in the reference's default double build
// (4 in a single-precision build; the reader takes either, by file size).
// The grid is not stored: it comes from the options, nx here.
int claire_b200_read_bin(const char* path, const int nx[3], float* data) {
  if (!path || !nx || !data || nx[0] < 1 || nx[1] < 1 || nx[2] < 1) return CB_ERR_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return CB_ERR_ARG;
  unsigned char hd[8];
  const bool hok = std::fread(hd, 1, 8, f) == 8;
  std::fseek(f, 0, SEEK_END);
  const long long size = std::ftell(f);
  std::fseek(f, 8, SEEK_SET);
  const long long n = (long long)nx[0] * nx[1] * nx[2];
  int rc = CB_OK;
  if (!hok || get<int>(hd, 0, true) != 1211214 || get<int>(hd, 4, true) != n) rc = CB_ERR_ARG;
  const long long per = (rc == CB_OK && n > 0) ? (size - 8) / n : 0;
  if (rc == CB_OK && ((size - 8) % n || (per != 8 && per != 4))) rc = CB_ERR_ARG;
  if (rc == CB_OK) {
    std::vector<unsigned char> raw((size_t)(n * per));
    if (std::fread(raw.data(), 1, raw.size(), f) != raw.size()) rc = CB_ERR_ARG;
    else if (per == 8) convert<double>(raw.data(), data, n, true);
    else convert<float>(raw.data(), data, n, true);
  }
  std::fclose(f);
  return rc;
}

int claire_b200_write_bin(const char* path, const int nx[3], const float* data) {
  if (!path || !nx || !data || nx[0] < 1 || nx[1] < 1 || nx[2] < 1) return CB_ERR_ARG;
  const long long n = (long long)nx[0] * nx[1] * nx[2];
  if (n > 2147483647LL) return CB_ERR_TOO_LARGE;
  std::vector<unsigned char> out((size_t)(8 + 8 * n));
  auto be32 = [&](size_t off, uint32_t v) {
    for (int i = 0; i < 4; ++i) out[off + i] = (unsigned char)(v >> (24 - 8 * i));
  };
  be32(0, 1211214u);
  be32(4, (uint32_t)n);
  for (long long i = 0; i < n; ++i) {
    uint64_t bits;
    const double v = (double)data[i];
    std::memcpy(&bits, &v, 8);
    for (int k = 0; k < 8; ++k) out[8 + 8 * i + k] = (unsigned char)(bits >> (56 - 8 * k));
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) return CB_ERR_ARG;
  const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
  return (std::fclose(f) == 0 && ok) ? CB_OK : CB_ERR_ARG;
}

int claire_b200_preprocess(float* m, const int nx[3], int rescale, const double sigma[3], void* stream) {
  if (!m || !nx || nx[0] < 1 || nx[1] < 1 || nx[2] < 1) return CB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const long long n = (long long)nx[0] * nx[1] * nx[2];
  if (rescale) {
    const int np = cb::field_stats_parts(n);
    double* parts = nullptr;
    if (cudaMallocAsync((void**)&parts, sizeof(double) * (3 * np + 2), s) != cudaSuccess) return CB_ERR_ALLOC;
    int e = cb::launch_field_stats(m, 0, n, 1, parts, s);
    if (!e) {
      k_minmax<<<1, 32, 0, s>>>(parts, np);
      k_normalize<<<148 * 4, 256, 0, s>>>(m, n, parts + 3 * np);
      e = (int)cudaGetLastError();
    }
    cudaFreeAsync(parts, s);
    if (e) return CB_ERR_CUDA;
  }
  if (sigma) {
    const int e = claire_b200_smooth(m, m, nx, sigma, stream);
    if (e) return e;
  }
  return cudaStreamSynchronize(s) == cudaSuccess ? CB_OK : CB_ERR_CUDA;
}

}  // extern "C"
