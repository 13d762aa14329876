// C ABI entry points (include/xtric.h): contexts, allocation, graph build,
// counting and the generators. Together they replace the reference's
// single-device engine TriangleCountingSingle (xxtric-gpu.hpp:27 constructor:
// copies the CSR to the device; :192 count(); :272 clear(): frees it) and
// its kernel launcher single_gpu_count (counting.cu:537-577).
#include <cmath>
#include <cstring>
#include <new>

#include "xt_internal.cuh"

namespace xt {

xt_status gen_rmat(Ctx *c, int scale, int64_t ne, uint64_t seed, int a16, int b16, int c16, int noise_pct,
                   int permute, int32_t *d_src, int32_t *d_dst);
xt_status gen_chunglu(Ctx *c, int64_t n, const uint64_t *cdf, int64_t ne, uint64_t seed, int permute,
                      int32_t *d_src, int32_t *d_dst);
xt_status gen_er(Ctx *c, int64_t n, int64_t ne, uint64_t seed, int32_t *d_src, int32_t *d_dst);
xt_status gen_rgg(Ctx *c, int64_t nv, int nprocs, double radius, int64_t cap, int64_t *n_pairs, int32_t *d_src,
                  int32_t *d_dst);

xt_status set_error(Ctx *c, xt_status s, const std::string &msg) {
  if (c) c->last_error = msg;
  return s;
}

xt_status cuda_status(Ctx *c, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return XT_OK;
  cudaGetLastError();  // clear a sticky launch error where possible
  xt_status s = (e == cudaErrorMemoryAllocation) ? XT_ERR_OOM : XT_ERR_CUDA;
  return set_error(c, s, std::string(what) + ": " + cudaGetErrorString(e));
}

xt_status dalloc(Ctx *c, void **p, size_t bytes) {
  *p = nullptr;
  if (c->fail_alloc_countdown > 0 && --c->fail_alloc_countdown == 0)
    return set_error(c, XT_ERR_OOM, "device allocation failed (injected by xt_debug_fail_alloc)");
  if (bytes == 0) bytes = 1;
  cudaError_t e = cudaMallocAsync(p, bytes, c->stream);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_error(c, XT_ERR_OOM,
                     "device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
  }
  c->live[*p] = bytes;
  c->bytes_live += int64_t(bytes);
  if (c->bytes_live > c->bytes_peak) c->bytes_peak = c->bytes_live;
  if (c->shared_live) {
    const int64_t v = c->shared_live->fetch_add(int64_t(bytes)) + int64_t(bytes);
    int64_t pk = c->shared_peak->load();
    while (v > pk && !c->shared_peak->compare_exchange_weak(pk, v)) {
    }
  }
  return XT_OK;
}

void dfree(Ctx *c, void *p) {
  if (!p) return;
  auto it = c->live.find(p);
  if (it != c->live.end()) {
    c->bytes_live -= int64_t(it->second);
    if (c->shared_live) c->shared_live->fetch_sub(int64_t(it->second));
    c->live.erase(it);
  }
  cudaFreeAsync(p, c->stream);
}

}  // namespace xt

using namespace xt;

extern "C" {

const char *xt_strerror(xt_status s) {
  switch (s) {
    case XT_OK: return "ok";
    case XT_ERR_INVALID: return "invalid argument";
    case XT_ERR_CUDA: return "CUDA error";
    case XT_ERR_OOM: return "out of device memory";
    case XT_ERR_IO: return "I/O error";
    case XT_ERR_OVERFLOW: return "size overflow";
    case XT_ERR_TIMEOUT: return "device wait timed out";
    case XT_ERR_ADMISSION: return "request exceeds the memory budget";
    case XT_ERR_NOT_READY: return "result not ready";
    case XT_ERR_NO_DEVICE: return "no usable CUDA device";
    case XT_ERR_CLOSED: return "closed";
  }
  return "unknown status";
}

const char *xt_last_error(const xt_ctx *ctx) { return ctx ? ctx->c.last_error.c_str() : "null context"; }

xt_status xt_open(int device, xt_ctx **out) {
  if (!out) return XT_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return XT_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) return XT_ERR_INVALID;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return XT_ERR_CUDA;
  if (prop.major < 10) return XT_ERR_NO_DEVICE;  // built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return XT_ERR_CUDA;
  xt_ctx *ctx = new (std::nothrow) xt_ctx();
  if (!ctx) return XT_ERR_OOM;
  Ctx *c = &ctx->c;
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  c->smem_optin = prop.sharedMemPerBlockOptin;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return XT_ERR_CUDA;
  }
  c->own_stream = true;
  // keep freed pool memory cached: graphs are rebuilt and counted repeatedly
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  if (cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess || cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    delete ctx;
    return XT_ERR_CUDA;
  }
  *out = ctx;
  return XT_OK;
}

xt_status xt_close(xt_ctx *ctx) {
  if (!ctx) return XT_ERR_INVALID;
  Ctx *c = &ctx->c;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaFree(c->d_err);
  if (c->copy_stream) {
    cudaStreamSynchronize(c->copy_stream);
    cudaStreamDestroy(c->copy_stream);
  }
  if (c->own_stream) cudaStreamDestroy(c->stream);
  delete ctx;
  return XT_OK;
}

xt_status xt_set_stream(xt_ctx *ctx, void *stream) {
  if (!ctx) return XT_ERR_INVALID;
  Ctx *c = &ctx->c;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  c->stream = static_cast<cudaStream_t>(stream);
  c->own_stream = false;
  return XT_OK;
}

xt_status xt_debug_fail_alloc(xt_ctx *ctx, int64_t k) {
  if (!ctx) return XT_ERR_INVALID;
  ctx->c.fail_alloc_countdown = k > 0 ? k : 0;
  return XT_OK;
}

int64_t xt_launch_count(const xt_ctx *ctx) { return ctx ? ctx->c.launches : -1; }

xt_status xt_mem_stats(xt_ctx *ctx, int64_t *live, int64_t *peak, int reset_peak) {
  if (!ctx) return XT_ERR_INVALID;
  Ctx *c = &ctx->c;
  if (live) *live = c->bytes_live;
  if (peak) *peak = c->bytes_peak;
  if (reset_peak) c->bytes_peak = c->bytes_live;
  return XT_OK;
}

static xt_status finish_build(xt_ctx *ctx, xt_graph *gr, xt_status s, xt_graph **out) {
  Ctx *c = &ctx->c;
  if (s == XT_OK) s = make_plan(&gr->g);
  if (s == XT_OK) s = cuda_status(c, cudaStreamSynchronize(c->stream), "build");
  if (s != XT_OK) {
    free_graph_device(&gr->g);
    cudaStreamSynchronize(c->stream);
    delete gr;
    return s;
  }
  *out = gr;
  return XT_OK;
}

xt_status xt_graph_from_device_edges(xt_ctx *ctx, int64_t nv, int64_t ne, const int32_t *d_src,
                                     const int32_t *d_dst, int orient, xt_graph **out) {
  if (!ctx || !out || (ne > 0 && (!d_src || !d_dst))) return XT_ERR_INVALID;
  *out = nullptr;
  Ctx *c = &ctx->c;
  cudaSetDevice(c->device);
  xt_graph *gr = new (std::nothrow) xt_graph();
  if (!gr) return XT_ERR_OOM;
  xt_status s = build_from_edges(c, nv, ne, d_src, d_dst, orient, &gr->g);
  return finish_build(ctx, gr, s, out);
}

xt_status xt_graph_from_edges(xt_ctx *ctx, int64_t nv, int64_t ne, const int32_t *src, const int32_t *dst,
                              int orient, xt_graph **out) {
  if (!ctx || !out || ne < 0 || (ne > 0 && (!src || !dst))) return XT_ERR_INVALID;
  *out = nullptr;
  Ctx *c = &ctx->c;
  cudaSetDevice(c->device);
  int32_t *ds = nullptr, *dd = nullptr;
  XT_TRY(dalloc_n(c, &ds, size_t(ne > 0 ? ne : 1)));
  xt_status s = dalloc_n(c, &dd, size_t(ne > 0 ? ne : 1));
  xt_graph *gr = nullptr;
  if (s == XT_OK) {
    gr = new (std::nothrow) xt_graph();
    if (!gr) s = XT_ERR_OOM;
  }
  if (s == XT_OK) {
    // the copy-in runs in chunks beside the first build step
    const HostRows up{src, dst};
    s = build_from_edges(c, nv, ne, ds, dd, orient, &gr->g, &up);
    s = finish_build(ctx, gr, s, out);
  }
  dfree(c, ds);
  dfree(c, dd);
  return s;
}

xt_status xt_graph_from_csr(xt_ctx *ctx, int64_t nv, const int64_t *offsets, const int64_t *tails, int flags,
                            int orient, xt_graph **out) {
  if (!ctx || !out || !offsets || nv < 1) return XT_ERR_INVALID;
  *out = nullptr;
  Ctx *c = &ctx->c;
  cudaSetDevice(c->device);
  // host-side header checks, as a reader of the vite layout would make
  if (offsets[0] != 0) return set_error(c, XT_ERR_INVALID, "offsets[0] must be 0");
  const int64_t ne = offsets[nv];
  if (ne < 0 || (ne > 0 && !tails)) return set_error(c, XT_ERR_INVALID, "bad offsets[nv] or null tails");
  int64_t *doff = nullptr, *dt = nullptr;
  XT_TRY(dalloc_n(c, &doff, size_t(nv + 1)));
  xt_status s = dalloc_n(c, &dt, size_t(ne > 0 ? ne : 1));
  if (s == XT_OK)
    s = cuda_status(c, cudaMemcpyAsync(doff, offsets, sizeof(int64_t) * (nv + 1), cudaMemcpyHostToDevice, c->stream),
                    "H2D");
  if (s == XT_OK && ne > 0)
    s = cuda_status(c, cudaMemcpyAsync(dt, tails, sizeof(int64_t) * ne, cudaMemcpyHostToDevice, c->stream), "H2D");
  xt_graph *gr = nullptr;
  if (s == XT_OK) {
    gr = new (std::nothrow) xt_graph();
    if (!gr) s = XT_ERR_OOM;
  }
  if (s == XT_OK) {
    s = build_from_csr(c, nv, doff, dt, (flags & XT_CSR_CANONICAL) != 0, orient, &gr->g);
    s = finish_build(ctx, gr, s, out);
  }
  dfree(c, doff);
  dfree(c, dt);
  cudaStreamSynchronize(c->stream);
  return s;
}

xt_status xt_graph_from_vite(xt_ctx *ctx, const char *path, int elem_bytes, int flags, int orient,
                             xt_graph **out) {
  if (!ctx || !out || !path) return XT_ERR_INVALID;
  *out = nullptr;
  Ctx *c = &ctx->c;
  cudaSetDevice(c->device);
  xt_graph *gr = new (std::nothrow) xt_graph();
  if (!gr) return XT_ERR_OOM;
  xt_status s = build_from_vite(c, path, elem_bytes, (flags & XT_CSR_CANONICAL) != 0, orient, &gr->g);
  return finish_build(ctx, gr, s, out);
}

xt_status xt_graph_get_info(const xt_graph *gr, xt_graph_info *info) {
  if (!gr || !info) return XT_ERR_INVALID;
  const Graph &g = gr->g;
  std::memset(info, 0, sizeof(*info));
  info->nv = g.nv;
  info->n_input = g.n_input;
  info->n_edges = g.ne;
  info->max_degree = g.max_degree;
  info->max_out_degree = g.max_out_degree;
  info->max_in_degree = g.max_in_degree;
  info->wedge_work = g.wedge_work;
  info->stream_work = g.stream_work;
  info->alg_bytes = 16 * (g.nv + 1) + 4 * g.ne + int64_t(sizeof(InRec)) * g.ne + 4 * g.stream_work;
  info->tail_alg_bytes = 8 * (g.nv + 1) + 4 * g.ne + 16 * g.ne + 4 * g.wedge_work;
  info->orient = g.orient;
  info->footprint_bytes = 16 * (g.nv + 1) + 4 * g.ne + int64_t(sizeof(InRec)) * g.ne + 4 * g.colp_len;
  info->cluster_tasks = cluster_task_count(&g);
  return XT_OK;
}

xt_status xt_graph_get_csr(const xt_graph *gr, int64_t *offsets, int32_t *cols) {
  if (!gr || !offsets || (gr->g.ne > 0 && !cols)) return XT_ERR_INVALID;
  const Graph &g = gr->g;
  Ctx *c = g.ctx;
  cudaSetDevice(c->device);
  XT_CUDA(c, cudaMemcpyAsync(offsets, g.d_off, sizeof(int64_t) * (g.nv + 1), cudaMemcpyDeviceToHost, c->stream));
  if (g.ne > 0)
    XT_CUDA(c, cudaMemcpyAsync(cols, g.d_col, sizeof(int32_t) * g.ne, cudaMemcpyDeviceToHost, c->stream));
  XT_CUDA(c, cudaStreamSynchronize(c->stream));
  return XT_OK;
}

xt_status xt_synchronize(xt_ctx *ctx) {
  if (!ctx) return XT_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  XT_CUDA(&ctx->c, cudaStreamSynchronize(ctx->c.stream));
  return XT_OK;
}

xt_status xt_graph_get_perm(const xt_graph *gr, int32_t *new_to_old) {
  if (!gr || !new_to_old) return XT_ERR_INVALID;
  const Graph &g = gr->g;
  Ctx *c = g.ctx;
  cudaSetDevice(c->device);
  if (g.d_perm) {
    XT_CUDA(c, cudaMemcpyAsync(new_to_old, g.d_perm, sizeof(int32_t) * g.nv, cudaMemcpyDeviceToHost, c->stream));
    XT_CUDA(c, cudaStreamSynchronize(c->stream));
  } else {
    for (int64_t i = 0; i < g.nv; i++) new_to_old[i] = int32_t(i);
  }
  return XT_OK;
}

xt_status xt_graph_free(xt_graph *gr) {
  if (!gr) return XT_ERR_INVALID;
  Ctx *c = gr->g.ctx;
  if (c) cudaSetDevice(c->device);
  free_graph_device(&gr->g);
  if (c) cudaStreamSynchronize(c->stream);
  delete gr;
  return XT_OK;
}

xt_status xt_count_async(xt_graph *gr, int64_t *d_global, int64_t *d_pv) {
  if (!gr || !d_global) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  return count_graph(&gr->g, d_global, d_pv);
}

xt_status xt_count(xt_graph *gr, int64_t *global, int64_t *per_vertex) {
  if (!gr || !global) return XT_ERR_INVALID;
  Graph &g = gr->g;
  Ctx *c = g.ctx;
  cudaSetDevice(c->device);
  int64_t *d = nullptr;
  XT_TRY(dalloc_n(c, &d, size_t(1 + (per_vertex ? g.nv : 0))));
  xt_status s = count_graph(&g, d, per_vertex ? d + 1 : nullptr);
  if (s == XT_OK)
    s = cuda_status(c, cudaMemcpyAsync(global, d, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream), "D2H");
  if (s == XT_OK && per_vertex)
    s = cuda_status(c, cudaMemcpyAsync(per_vertex, d + 1, sizeof(int64_t) * g.nv, cudaMemcpyDeviceToHost, c->stream),
                    "D2H");
  dfree(c, d);
  if (s == XT_OK) s = cuda_status(c, cudaStreamSynchronize(c->stream), "count");
  if (s == XT_OK) s = count_status(c);
  return s;
}

xt_status xt_count_edges(xt_graph *gr, int64_t *global, int64_t *support) {
  if (!gr || !global || !support) return XT_ERR_INVALID;
  Graph &g = gr->g;
  Ctx *c = g.ctx;
  cudaSetDevice(c->device);
  int64_t *d = nullptr;
  XT_TRY(dalloc_n(c, &d, size_t(1 + g.ne)));
  xt_status s = count_graph(&g, d, nullptr, nullptr, d + 1);
  if (s == XT_OK)
    s = cuda_status(c, cudaMemcpyAsync(global, d, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream), "D2H");
  if (s == XT_OK && g.ne > 0)
    s = cuda_status(c, cudaMemcpyAsync(support, d + 1, sizeof(int64_t) * g.ne, cudaMemcpyDeviceToHost, c->stream),
                    "D2H");
  dfree(c, d);
  if (s == XT_OK) s = cuda_status(c, cudaStreamSynchronize(c->stream), "count");
  if (s == XT_OK) s = count_status(c);
  return s;
}

xt_status xt_count_edges_async(xt_graph *gr, int64_t *d_global, int64_t *d_support) {
  if (!gr || !d_global || (gr->g.ne > 0 && !d_support)) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  return count_graph(&gr->g, d_global, nullptr, nullptr, d_support);
}

xt_status xt_count_shard_async(xt_graph *gr, int shard, int nshards, int64_t *d_global, int64_t *d_pv) {
  if (!gr || !d_global) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  return count_graph(&gr->g, d_global, d_pv, nullptr, nullptr, shard, nshards);
}

xt_status xt_count_edges_shard_async(xt_graph *gr, int shard, int nshards, int64_t *d_global, int64_t *d_support) {
  if (!gr || !d_global || (gr->g.ne > 0 && !d_support)) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  return count_graph(&gr->g, d_global, nullptr, nullptr, d_support, shard, nshards);
}

xt_status xt_count_device(int64_t nv, const int64_t *d_indices, const int64_t *d_edge_list, int64_t *d_count,
                          int accumulate, void *stream) {
  if (nv < 1 || !d_indices || !d_count) return XT_ERR_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return XT_ERR_NO_DEVICE;
  // a transient context on the caller's device and stream
  xt_ctx *ctx = nullptr;
  XT_TRY(xt_open(dev, &ctx));
  Ctx *c = &ctx->c;
  cudaStreamDestroy(c->stream);
  c->stream = static_cast<cudaStream_t>(stream);
  c->own_stream = false;
  Graph g;
  xt_status s = build_from_csr(c, nv, d_indices, d_edge_list, true, XT_ORIENT_DEGREE, &g);
  int64_t *tmp = nullptr;
  if (s == XT_OK) s = make_plan(&g);
  if (s == XT_OK) s = dalloc_n(c, &tmp, 1);
  if (s == XT_OK) s = count_graph(&g, tmp, nullptr);
  if (s == XT_OK && accumulate) {
    int64_t h = 0, add = 0;
    s = cuda_status(c, cudaMemcpyAsync(&h, d_count, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream), "D2H");
    if (s == XT_OK)
      s = cuda_status(c, cudaMemcpyAsync(&add, tmp, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream), "D2H");
    if (s == XT_OK) s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync");
    h += add;
    if (s == XT_OK)
      s = cuda_status(c, cudaMemcpyAsync(d_count, &h, sizeof(int64_t), cudaMemcpyHostToDevice, c->stream), "H2D");
  } else if (s == XT_OK) {
    s = cuda_status(c, cudaMemcpyAsync(d_count, tmp, sizeof(int64_t), cudaMemcpyDeviceToDevice, c->stream), "D2D");
  }
  dfree(c, tmp);
  free_graph_device(&g);
  cudaStreamSynchronize(c->stream);
  c->stream = nullptr;
  cudaFree(c->d_err);
  delete ctx;
  return s;
}

xt_status xt_gen_rmat(xt_ctx *ctx, int scale, int64_t ne, uint64_t seed, int a16, int b16, int c16, int noise_pct,
                      int permute, int32_t *d_src, int32_t *d_dst) {
  if (!ctx) return XT_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  return gen_rmat(&ctx->c, scale, ne, seed, a16, b16, c16, noise_pct, permute, d_src, d_dst);
}

xt_status xt_gen_chunglu(xt_ctx *ctx, int64_t n, const uint64_t *cdf, int64_t ne, uint64_t seed, int permute,
                         int32_t *d_src, int32_t *d_dst) {
  if (!ctx) return XT_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  return gen_chunglu(&ctx->c, n, cdf, ne, seed, permute, d_src, d_dst);
}

xt_status xt_gen_er(xt_ctx *ctx, int64_t n, int64_t ne, uint64_t seed, int32_t *d_src, int32_t *d_dst) {
  if (!ctx) return XT_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  return gen_er(&ctx->c, n, ne, seed, d_src, d_dst);
}

xt_status xt_gen_rgg(xt_ctx *ctx, int64_t nv, int nprocs, double radius, int64_t cap, int64_t *n_pairs,
                     int32_t *d_src, int32_t *d_dst) {
  if (!ctx) return XT_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  return gen_rgg(&ctx->c, nv, nprocs, radius, cap, n_pairs, d_src, d_dst);
}

xt_status xt_graph_from_rgg(xt_ctx *ctx, int64_t nv, int nprocs, double radius, int orient, xt_graph **out) {
  if (!ctx || !out) return XT_ERR_INVALID;
  *out = nullptr;
  Ctx *c = &ctx->c;
  cudaSetDevice(c->device);
  int64_t m = 0;
  XT_TRY(gen_rgg(c, nv, nprocs, radius, 0, &m, nullptr, nullptr));
  int32_t *ds = nullptr, *dd = nullptr;
  XT_TRY(dalloc_n(c, &ds, size_t(m > 0 ? m : 1)));
  xt_status s = dalloc_n(c, &dd, size_t(m > 0 ? m : 1));
  if (s == XT_OK && m > 0) s = gen_rgg(c, nv, nprocs, radius, m, &m, ds, dd);
  xt_graph *gr = nullptr;
  if (s == XT_OK) {
    gr = new (std::nothrow) xt_graph();
    if (!gr) s = XT_ERR_OOM;
  }
  if (s == XT_OK) {
    s = build_from_edges(c, nv, m, ds, dd, orient, &gr->g);
    if (s == XT_OK) gr->g.n_input = 2 * m;  // the reference's directed entries
    s = finish_build(ctx, gr, s, out);
  }
  dfree(c, ds);
  dfree(c, dd);
  cudaStreamSynchronize(c->stream);
  return s;
}

int64_t xt_chunglu_cdf(int64_t n, double gamma, double mean_deg, double max_deg, uint64_t *cdf) {
  // expected degree w_i = max_deg * (1 + i/i0)^(-1/(gamma-1)); i0 by
  // bisection so that the integral approximation of the mean of w,
  // (max_deg/n) * int_0^n (1 + x/i0)^(-alpha) dx, equals mean_deg; weights
  // in 1/1024 units (at least 1) so the device draws with integers only
  if (n < 1 || !cdf || gamma <= 1.0 || mean_deg <= 0 || max_deg <= 0) return -1;
  const double alpha = 1.0 / (gamma - 1.0);
  double lo = 1e-9, hi = double(n);
  for (int it = 0; it < 200; it++) {
    double i0 = 0.5 * (lo + hi), integral;
    if (std::fabs(1.0 - alpha) < 1e-12) integral = i0 * std::log(1.0 + double(n) / i0);
    else integral = i0 / (1.0 - alpha) * (std::pow(1.0 + double(n) / i0, 1.0 - alpha) - 1.0);
    if (max_deg * integral / double(n) > mean_deg) hi = i0;
    else lo = i0;
  }
  const double i0 = 0.5 * (lo + hi);
  cdf[0] = 0;
  for (int64_t i = 0; i < n; i++) {
    double w = max_deg * std::pow(1.0 + double(i) / i0, -alpha);
    uint64_t W = uint64_t(std::llround(w * 1024.0));
    if (W < 1) W = 1;
    cdf[i + 1] = cdf[i] + W;
  }
  return int64_t(std::llround(double(n) * mean_deg / 2.0));
}

}  // extern "C"
