// The vite binary graph file read into the device builder.
//
// Replaces BinaryEdgeList::read (graph.hpp:294-395) for one process, whose
// host pass copies every {tail, weight} record into host Edge objects. Here
// the host only streams the file's bytes: chunks are read into two pinned
// staging buffers in turn and copied to the device, where a kernel takes the
// tails out of the records (the weights are skipped; the count ignores
// them), so reading chunk i + 1 from the file overlaps the copy and parse of
// chunk i. Layout: [nv][ne][offsets: nv+1][ne x {tail, weight}] with 8-byte
// fields, or 4-byte fields for USE_32_BIT_GRAPH (deftypes.hpp:40-49). The
// file size must match the header exactly; the offsets are checked on the
// device by the CSR builder (monotone, within [0, ne]) and here for
// offsets[0] = 0 and offsets[nv] = ne.
#include <stdio.h>

#include <algorithm>

#include "xt_internal.cuh"

namespace xt {

// records of a chunk -> their tails (int64), at the chunk's place in tails
template <int EB>
__global__ void k_vite_tails(const unsigned char *__restrict__ buf, int64_t k, int64_t *__restrict__ tails) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < k; i += int64_t(gridDim.x) * blockDim.x) {
    if (EB == 8) tails[i] = reinterpret_cast<const int64_t *>(buf)[2 * i];
    else tails[i] = int64_t(reinterpret_cast<const int32_t *>(buf)[2 * i]);
  }
}

// 4-byte offsets -> int64
__global__ void k_vite_widen(const int32_t *__restrict__ in, int64_t n, int64_t *__restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = int64_t(in[i]);
}

namespace {

struct HostFile {
  FILE *f = nullptr;
  ~HostFile() {
    if (f) fclose(f);
  }
};

bool read_full(FILE *f, void *dst, size_t bytes) {
  char *p = static_cast<char *>(dst);
  while (bytes) {
    const size_t k = fread(p, 1, bytes, f);
    if (k == 0) return false;
    p += k;
    bytes -= k;
  }
  return true;
}

unsigned vite_grid(const Ctx *c, int64_t n) {
  int64_t g = (n + 255) / 256, cap = int64_t(c->sm_count) * 16;
  return unsigned(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace

// Streams `bytes` of the open file into device memory dst (or, with parse,
// through the record parser into tails), chunk by chunk through two pinned
// staging buffers.
static xt_status stream_file(Ctx *c, FILE *f, int64_t bytes, unsigned char *dst, int eb, int64_t *tails,
                             unsigned char *stage[2], unsigned char *dstage[2], cudaEvent_t ev[2], int64_t chunk) {
  const int64_t rec = 2 * int64_t(eb);
  for (int64_t done = 0, i = 0; done < bytes; i++) {
    const int b = int(i & 1);
    int64_t k = std::min(chunk, bytes - done);
    if (tails) k -= k % rec;  // whole records per chunk
    XT_CUDA(c, cudaEventSynchronize(ev[b]));  // the buffer's previous copy has finished
    if (!read_full(f, stage[b], size_t(k))) return set_error(c, XT_ERR_IO, "vite: short read");
    if (!tails) {
      XT_CUDA(c, cudaMemcpyAsync(dst + done, stage[b], size_t(k), cudaMemcpyHostToDevice, c->stream));
    } else {
      XT_CUDA(c, cudaMemcpyAsync(dstage[b], stage[b], size_t(k), cudaMemcpyHostToDevice, c->stream));
      const int64_t nrec = k / rec, first = done / rec;
      if (eb == 8)
        k_vite_tails<8><<<counted(c, vite_grid(c, nrec)), 256, 0, c->stream>>>(dstage[b], nrec, tails + first);
      else
        k_vite_tails<4><<<counted(c, vite_grid(c, nrec)), 256, 0, c->stream>>>(dstage[b], nrec, tails + first);
      XT_CUDA(c, cudaGetLastError());
    }
    XT_CUDA(c, cudaEventRecord(ev[b], c->stream));
    done += k;
  }
  return XT_OK;
}

xt_status build_from_vite(Ctx *c, const char *path, int eb, bool canonical, int orient, Graph *g) {
  if (!path || (eb != 8 && eb != 4)) return set_error(c, XT_ERR_INVALID, "vite: bad arguments");
  HostFile hf;
  hf.f = fopen(path, "rb");
  if (!hf.f) return set_error(c, XT_ERR_IO, std::string("vite: cannot open ") + path);
  int64_t hdr[2] = {0, 0};
  if (eb == 8) {
    if (!read_full(hf.f, hdr, sizeof(hdr))) return set_error(c, XT_ERR_IO, "vite: short header");
  } else {
    int32_t h32[2];
    if (!read_full(hf.f, h32, sizeof(h32))) return set_error(c, XT_ERR_IO, "vite: short header");
    hdr[0] = h32[0];
    hdr[1] = h32[1];
  }
  const int64_t nv = hdr[0], ne = hdr[1];
  if (nv < 1 || ne < 0) return set_error(c, XT_ERR_IO, "vite: bad header");
  if (fseeko(hf.f, 0, SEEK_END) != 0) return set_error(c, XT_ERR_IO, "vite: seek");
  const int64_t size = ftello(hf.f);
  if (size != 2 * eb + (nv + 1) * eb + ne * 2 * eb)
    return set_error(c, XT_ERR_IO, "vite: the file size does not match its header");
  if (fseeko(hf.f, 2 * eb, SEEK_SET) != 0) return set_error(c, XT_ERR_IO, "vite: seek");
  constexpr int64_t kChunk = int64_t(64) << 20;
  unsigned char *stage[2] = {nullptr, nullptr}, *dstage[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int64_t *d_off = nullptr, *d_tails = nullptr;
  int32_t *off32 = nullptr;
  xt_status s = XT_OK;
  do {
    for (int b = 0; b < 2 && s == XT_OK; b++) {
      s = cuda_status(c, cudaHostAlloc(reinterpret_cast<void **>(&stage[b]), size_t(kChunk), cudaHostAllocDefault),
                      "pinned staging");
      if (s == XT_OK) s = dalloc_n(c, &dstage[b], size_t(kChunk));
      if (s == XT_OK) s = cuda_status(c, cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming), "event");
      if (s == XT_OK) s = cuda_status(c, cudaEventRecord(ev[b], c->stream), "event");
    }
    if (s != XT_OK) break;
    if ((s = dalloc_n(c, &d_off, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_tails, size_t(ne > 0 ? ne : 1))) != XT_OK) break;
    if (eb == 8) {
      s = stream_file(c, hf.f, (nv + 1) * 8, reinterpret_cast<unsigned char *>(d_off), 8, nullptr, stage, dstage,
                      ev, kChunk);
    } else {
      if ((s = dalloc_n(c, &off32, size_t(nv + 1))) != XT_OK) break;
      s = stream_file(c, hf.f, (nv + 1) * 4, reinterpret_cast<unsigned char *>(off32), 4, nullptr, stage, dstage,
                      ev, kChunk);
      if (s == XT_OK) {
        k_vite_widen<<<counted(c, vite_grid(c, nv + 1)), 256, 0, c->stream>>>(off32, nv + 1, d_off);
        s = cuda_status(c, cudaGetLastError(), "vite offsets");
      }
    }
    if (s != XT_OK) break;
    if (ne > 0 && (s = stream_file(c, hf.f, ne * 2 * eb, nullptr, eb, d_tails, stage, dstage, ev, kChunk)) != XT_OK)
      break;
    int64_t ends[2] = {-1, -1};
    s = cuda_status(c, cudaMemcpyAsync(&ends[0], d_off, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream), "D2H");
    if (s == XT_OK)
      s = cuda_status(c, cudaMemcpyAsync(&ends[1], d_off + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream),
                      "D2H");
    if (s == XT_OK) s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync");
    if (s == XT_OK && (ends[0] != 0 || ends[1] != ne))
      s = set_error(c, XT_ERR_IO, "vite: offsets[0] must be 0 and offsets[nv] must be ne");
    if (s == XT_OK) s = build_from_csr(c, nv, d_off, d_tails, canonical, orient, g);
  } while (0);
  cudaStreamSynchronize(c->stream);  // no copy reads a staging buffer after it is freed
  for (int b = 0; b < 2; b++) {
    if (stage[b]) cudaFreeHost(stage[b]);
    dfree(c, dstage[b]);
    if (ev[b]) cudaEventDestroy(ev[b]);
  }
  dfree(c, off32);
  dfree(c, d_off);
  dfree(c, d_tails);
  return s;
}

}  // namespace xt
