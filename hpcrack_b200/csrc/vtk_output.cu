// VTK XML ImageData output of one field of one level (vtk_output.cpp: write_total_de, write_total_u,
// write_total_H), written from the device-resident hierarchy without a double-precision copy to
// the host.
//
// The reference converts the field to a dense Float32 array on the host, base64-encodes it
// (vtk_base64_utilities.cpp) and writes the .vti piece plus the .pvti index.  Here one kernel on
// the context's stream converts and encodes in a single pass over the field (each thread turns 3
// Float32 values, 12 bytes, into 16 base64 characters), the characters are copied to pinned host
// memory on a copy stream, and a host thread writes both files once the copy has landed - so the
// next increment's kernels run while the D2H copy and the file writes proceed.  The bytes written
// are the reference's: the same XML text, the same Float32 rounding of the same values, the same
// base64 alphabet and padding, the same 4-byte length header encoded on its own.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>

#include "device_common.cuh"
#include "internal.h"

namespace hpc {
namespace {

enum VtkKind { VTK_SCALAR = 0, VTK_VECTOR = 1, VTK_CELL = 2 };

const char kB64[65] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

// The base64 alphabet (A-Z a-z 0-9 + /) by arithmetic: no table lookups in the kernel.
__device__ __forceinline__ unsigned b64c(unsigned v) {
  return v < 26 ? 'A' + v : v < 52 ? 'a' + (v - 26) : v < 62 ? '0' + (v - 52) : v == 62 ? '+' : '/';
}

struct VtkArgs {
  LevelGeo g;
  const double* src;  // scalar field, or component 0 of a vector field (components n apart)
  double scale;       // vector fields: the reference writes (float)(u_proportion * u)
  long long nvals;    // Float32 values in the stream
  long long ntrip;    // ceil(nvals / 3): one thread per 3 values
  char* out;          // 4 * ceil(4 nvals / 3) characters
};

// Value q of the dense Float32 stream, x fastest: nodes (S), interleaved components of nodes (V),
// elements (C) - the loops of write_scalar, write_vector and write_celltdata_H.
template <int KIND>
__device__ __forceinline__ float stream_value(const VtkArgs& a, long long q) {
  const LevelGeo& g = a.g;
  if (KIND == VTK_VECTOR) {
    const long long node = q / 3;
    const int m = (int)(q - node * 3);
    const int i = (int)(node % g.nx);
    const long long r = node / g.nx;
    const int j = (int)(r % g.ny), k = (int)(r / g.ny);
    const double v = a.src[(long long)m * g.n + i + (long long)j * g.px + (long long)k * g.plane];
    return __double2float_rn(__dmul_rn(a.scale, v));
  } else {
    const int nx = KIND == VTK_CELL ? g.nx - 1 : g.nx, ny = KIND == VTK_CELL ? g.ny - 1 : g.ny;
    const int i = (int)(q % nx);
    const long long r = q / nx;
    const int j = (int)(r % ny), k = (int)(r / ny);
    return __double2float_rn(a.src[i + (long long)j * g.px + (long long)k * g.plane]);
  }
}

__device__ __forceinline__ unsigned pack4(unsigned c0, unsigned c1, unsigned c2, unsigned c3) {
  return c0 | (c1 << 8) | (c2 << 16) | (c3 << 24);
}
// 3 bytes -> 4 characters, as one little-endian word of the output
__device__ __forceinline__ unsigned enc3(unsigned b0, unsigned b1, unsigned b2) {
  return pack4(b64c(b0 >> 2), b64c(((b0 << 4) & 0x30) | (b1 >> 4)), b64c(((b1 << 2) & 0x3C) | (b2 >> 6)),
               b64c(b2 & 0x3F));
}

template <int KIND>
__global__ void __launch_bounds__(256) vtk_pack_kernel(VtkArgs a) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < a.ntrip; t += stride) {
    const long long q0 = 3 * t;
    const int cnt = (int)min(3LL, a.nvals - q0);
    unsigned w[3] = {0u, 0u, 0u};
    for (int i = 0; i < cnt; ++i) w[i] = __float_as_uint(stream_value<KIND>(a, q0 + i));
    unsigned char b[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) b[i] = (unsigned char)(w[i >> 2] >> (8 * (i & 3)));
    unsigned* o = reinterpret_cast<unsigned*>(a.out + 16 * t);
    if (cnt == 3) {
      uint4 v;
      v.x = enc3(b[0], b[1], b[2]);
      v.y = enc3(b[3], b[4], b[5]);
      v.z = enc3(b[6], b[7], b[8]);
      v.w = enc3(b[9], b[10], b[11]);
      *reinterpret_cast<uint4*>(o) = v;
    } else if (cnt == 2) {  // 8 bytes: two triplets and a pair (one '=')
      o[0] = enc3(b[0], b[1], b[2]);
      o[1] = enc3(b[3], b[4], b[5]);
      o[2] = pack4(b64c(b[6] >> 2), b64c(((b[6] << 4) & 0x30) | (b[7] >> 4)), b64c((b[7] << 2) & 0x3C), '=');
    } else {  // 4 bytes: one triplet and a single byte (two '=')
      o[0] = enc3(b[0], b[1], b[2]);
      o[1] = pack4(b64c(b[3] >> 2), b64c((b[3] << 4) & 0x30), '=', '=');
    }
  }
}

// Host base64 of a few bytes (the 4-byte length header the reference encodes on its own).
std::string b64_host(const unsigned char* p, size_t n) {
  std::string s;
  size_t i = 0;
  for (; i + 3 <= n; i += 3) {
    s += kB64[p[i] >> 2];
    s += kB64[((p[i] << 4) & 0x30) | (p[i + 1] >> 4)];
    s += kB64[((p[i + 1] << 2) & 0x3C) | (p[i + 2] >> 6)];
    s += kB64[p[i + 2] & 0x3F];
  }
  if (n - i == 2) {
    s += kB64[p[i] >> 2];
    s += kB64[((p[i] << 4) & 0x30) | (p[i + 1] >> 4)];
    s += kB64[(p[i + 1] << 2) & 0x3C];
    s += '=';
  } else if (n - i == 1) {
    s += kB64[p[i] >> 2];
    s += kB64[(p[i] << 4) & 0x30];
    s += "==";
  }
  return s;
}

std::string fmt(const char* f, ...) __attribute__((format(printf, 1, 2)));
std::string fmt(const char* f, ...) {
  char buf[4096];
  va_list ap;
  va_start(ap, f);
  vsnprintf(buf, sizeof buf, f, ap);
  va_end(ap);
  return buf;
}

// One write in flight: the file texts around the encoded payload, and the thread that writes them.
struct VtkJob {
  std::thread th;
  int status = HPC_OK;
  std::string msg;
  std::string vti_path, pvti_path, prefix, suffix, pvti;
  const char* payload = nullptr;
  size_t payload_len = 0;
  cudaEvent_t copied = nullptr;
  int device = 0;

  void run() {
    cudaSetDevice(device);
    const cudaError_t e = cudaEventSynchronize(copied);
    if (e != cudaSuccess) {
      status = HPC_ERR_CUDA;
      msg = std::string("vtk copy: ") + cudaGetErrorString(e);
      return;
    }
    FILE* f = fopen(vti_path.c_str(), "wb+");
    if (!f) {
      status = HPC_ERR_IO;
      msg = "cannot open " + vti_path;
      return;
    }
    bool ok = fwrite(prefix.data(), 1, prefix.size(), f) == prefix.size();
    ok = ok && fwrite(payload, 1, payload_len, f) == payload_len;
    ok = ok && fwrite(suffix.data(), 1, suffix.size(), f) == suffix.size();
    ok = (fclose(f) == 0) && ok;
    FILE* p = ok ? fopen(pvti_path.c_str(), "wb+") : nullptr;
    if (p) {
      ok = fwrite(pvti.data(), 1, pvti.size(), p) == pvti.size();
      ok = (fclose(p) == 0) && ok;
    } else {
      ok = false;
    }
    if (!ok) {
      status = HPC_ERR_IO;
      msg = "cannot write " + (p ? pvti_path : vti_path);
    }
  }
};

int bad_arg(const char* msg) {
  set_error(msg);
  return HPC_ERR_ARG;
}

int join_job(hpc_ctx* c) {
  VtkJob* j = static_cast<VtkJob*>(c->vtk.job);
  if (!j) return HPC_OK;
  j->th.join();
  const int st = j->status;
  if (st != HPC_OK) set_error(j->msg);
  delete j;
  c->vtk.job = nullptr;
  return st;
}

}  // namespace

int vtk_release(hpc_ctx* c) {
  const int st = join_job(c);
  hpc_ctx::Vtk& v = c->vtk;
  if (v.dev) cudaFree(v.dev);
  if (v.host) cudaFreeHost(v.host);
  if (v.packed) cudaEventDestroy(v.packed);
  if (v.copied) cudaEventDestroy(v.copied);
  if (v.stream) cudaStreamDestroy(v.stream);
  v = hpc_ctx::Vtk{};
  return st;
}

}  // namespace hpc

using namespace hpc;

extern "C" int hpc_vtk_write(hpc_ctx* c, const char* option, int field, int level, double scale,
                             const char* filename, const char* field_name, int t) {
  if (!c || !option || !filename || !field_name) return bad_arg("null argument");
  const std::string opt(option);
  const int kind = opt == "S" ? VTK_SCALAR : opt == "V" ? VTK_VECTOR : opt == "C" ? VTK_CELL : -1;
  if (kind < 0) return bad_arg("vtk option must be \"S\", \"V\" or \"C\"");
  if (level < 0 || level > c->maxlevel) return bad_arg("bad level");
  const double* src = kind == VTK_VECTOR ? vector_field(c, field, level) : scalar_field(c, field, level);
  if (!src) return bad_arg(kind == VTK_VECTOR ? "option \"V\" needs a vector field" : "needs a scalar field");
  HPC_CUDA(cudaSetDevice(c->device));
  // the previous write owns the buffers until its thread is done
  if (const int st = join_job(c)) return st;

  const LevelGeo& g = c->L[level];
  const long long nodes = (long long)g.nx * g.ny * g.nz;
  const long long nvals = kind == VTK_VECTOR ? 3 * nodes
                          : kind == VTK_CELL ? (long long)(g.nx - 1) * (g.ny - 1) * (g.nz - 1)
                                             : nodes;
  const long long ntrip = (nvals + 2) / 3;
  const size_t chars = 4 * (size_t)((4 * nvals + 2) / 3);
  hpc_ctx::Vtk& v = c->vtk;
  if (!v.stream) {
    HPC_CUDA(cudaStreamCreateWithFlags(&v.stream, cudaStreamNonBlocking));
    HPC_CUDA(cudaEventCreateWithFlags(&v.packed, cudaEventDisableTiming));
    HPC_CUDA(cudaEventCreateWithFlags(&v.copied, cudaEventDisableTiming));
  }
  const size_t need = (size_t)ntrip * 16;  // whole 16-character groups (the tail thread writes fewer)
  if (v.cap < need) {
    if (v.dev) cudaFree(v.dev);
    if (v.host) cudaFreeHost(v.host);
    v.dev = nullptr;
    v.host = nullptr;
    v.cap = 0;
    HPC_CUDA(cudaMalloc((void**)&v.dev, need));
    HPC_CUDA(cudaMallocHost((void**)&v.host, need));
    v.cap = need;
  }
  if (nvals > 0) {
    VtkArgs a{g, src, scale, nvals, ntrip, v.dev};
    const int grid = (int)std::min<long long>((ntrip + 255) / 256, 148LL * 16);
    if (kind == VTK_VECTOR)
      vtk_pack_kernel<VTK_VECTOR><<<grid, 256, 0, c->stream>>>(a);
    else if (kind == VTK_CELL)
      vtk_pack_kernel<VTK_CELL><<<grid, 256, 0, c->stream>>>(a);
    else
      vtk_pack_kernel<VTK_SCALAR><<<grid, 256, 0, c->stream>>>(a);
    HPC_CHECK_LAUNCH(c);
  }
  HPC_CUDA(cudaEventRecord(v.packed, c->stream));
  HPC_CUDA(cudaStreamWaitEvent(v.stream, v.packed, 0));
  if (chars > 0) HPC_CUDA(cudaMemcpyAsync(v.host, v.dev, chars, cudaMemcpyDeviceToHost, v.stream));
  HPC_CUDA(cudaEventRecord(v.copied, v.stream));

  // File texts: write_header / write_pointdata_head / write_celltdata_H / write_end / write_pvtk of
  // vtk_output.cpp:26-446 for one rank (myid 0, one piece covering the level).
  const int ii = g.nx - 1, jj = g.ny - 1, kk = g.nz - 1;
  const double x0 = c->box[0], y0 = c->box[2], z0 = c->box[4];
  VtkJob* j = new VtkJob();
  j->device = c->device;
  j->copied = v.copied;
  j->payload = v.host;
  j->payload_len = chars;
  j->vti_path = std::strstr(filename, ".vti") ? std::string(filename)
                                              : fmt("Output/%s_l_%d_t_%d_Proc_%d.vti", filename, level, t, 0);
  j->pvti_path = std::strstr(filename, ".pvti") ? std::string(filename)
                                                : fmt("Output/%s_l_%d_t_%d.pvti", filename, level, t);
  std::string& s = j->prefix;
  s = "<?xml version=\"1.0\"?>\n";
  s += "<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
  s += fmt("<ImageData WholeExtent=\"%d %d %d %d %d %d \" \t\t\t\tOrigin=\"%f %f %f\" Spacing=\"%f %f %f\">\n", 0, ii,
           0, jj, 0, kk, x0, y0, z0, g.hx, g.hy, g.hz);
  s += fmt("<Piece Extent=\"%d %d %d %d %d %d\" >\n", 0, ii, 0, jj, 0, kk);
  if (kind == VTK_SCALAR) {
    s += fmt("<PointData Scalars=\"%s\">\n", field_name);
    s += fmt("<DataArray Name=\"%s\" type=\"Float32\" NumberOfComponents=\"1\" format=\"binary\">\n", field_name);
  } else if (kind == VTK_VECTOR) {
    s += fmt("<PointData Vectors=\"%s\">\n", field_name);
    s += fmt("<DataArray Name=\"%s\" type=\"Float32\" NumberOfComponents=\"3\" format=\"binary\">\n", field_name);
  } else {
    s += "<PointData></PointData>\n";
    s += fmt("<CellData Scalar = \"%s\">\n", field_name);
    s += fmt("<DataArray Name=\"%s\" type=\"Float32\" NumberOfComponents=\"1\" format=\"binary\">\n", field_name);
  }
  // the byte count, encoded as its own base64 block: the low 4 bytes of a little-endian long
  const long bytes = (long)(nvals * 4);
  unsigned char hdr[4];
  std::memcpy(hdr, &bytes, 4);
  s += b64_host(hdr, 4);
  j->suffix = kind == VTK_CELL ? "\n</DataArray>\n</CellData>\n</Piece>\n</ImageData>\n</VTKFile>"
                               : "\n</DataArray>\n</PointData>\n<CellData></CellData>\n</Piece>\n</ImageData>\n</VTKFile>";
  std::string& p = j->pvti;
  p = "<?xml version=\"1.0\"?>\n";
  p += "<VTKFile type=\"PImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
  p += fmt("<PImageData WholeExtent=\"0 %ld 0 %ld 0 %ld \" \t\t\t\tGhostLevel=\"0\" Origin=\"%f %f %f\" "
           "Spacing=\"%f %f %f\">\n",
           (long)ii, (long)jj, (long)kk, x0, y0, z0, g.hx, g.hy, g.hz);
  if (kind == VTK_SCALAR) {
    p += fmt("<PPointData Scalars=\"%s\">\n", field_name);
    p += fmt("<PDataArray Name=\"%s\" type=\"Float32\" NumberOfComponents=\"1\"/>\n", field_name);
  } else if (kind == VTK_VECTOR) {
    p += fmt("<PPointData Vectors=\"%s\">\n", field_name);
    p += fmt("<PDataArray Name=\"%s\" type=\"Float32\" NumberOfComponents=\"3\"/>\n", field_name);
  }
  if (kind == VTK_CELL) {
    p += "<PPointData></PPointData>\n";
    p += fmt("<PCellData Scalar = \"%s\">\n", field_name);
    p += fmt("<PDataArray Name=\"%s\" type=\"Float32\" NumberOfComponents=\"1\"/>\n", field_name);
    p += "</PCellData>\n";
  } else {
    p += "</PPointData>\n";
    p += "<PCellData></PCellData>\n";
  }
  p += fmt("<Piece Extent=\"%d %d %d %d %d %d\" Source=\"%s_l_%d_t_%d_Proc_%d.vti\"/>\n", 0, ii, 0, jj, 0, kk,
           filename, level, t, 0);
  p += "</PImageData>\n";
  p += "</VTKFile>\n";
  try {
    j->th = std::thread([j] { j->run(); });
  } catch (const std::exception& e) {
    delete j;
    HPC_CUDA(cudaEventSynchronize(v.copied));
    set_error(std::string("vtk writer thread: ") + e.what());
    return HPC_ERR_IO;
  }
  c->vtk.job = j;
  return HPC_OK;
}

extern "C" int hpc_vtk_wait(hpc_ctx* c) {
  if (!c) return bad_arg("null context");
  return join_job(c);
}
