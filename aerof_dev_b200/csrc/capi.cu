// capi.cu -- context lifetime, stream selection and host/device staging of
// the C ABI declared in include/aerof_gpu.h.
#include <cstring>

#include "common.cuh"

namespace aerof {

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

const double* in_dev(aerof_gpu_ctx* c, const double* p, size_t count, DBuf<double>& stage) {
  if (is_device_ptr(p)) return p;
  stage.ensure(count);
  AEROF_CUDA(cudaMemcpyAsync(stage.p, p, count * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return stage.p;
}

double* out_dev(aerof_gpu_ctx* c, double* p, size_t count, DBuf<double>& stage) {
  (void)c;
  if (is_device_ptr(p)) return p;
  stage.ensure(count);
  return stage.p;
}

void out_finish(aerof_gpu_ctx* c, double* user, const double* dev, size_t count) {
  if (user != dev)
    AEROF_CUDA(cudaMemcpyAsync(user, dev, count * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AEROF_CUDA(cudaStreamSynchronize(c->stream));
}

// Only the outermost scope records: a scope opened inside another one
// (a preconditioner apply inside the Gram-Schmidt scope, say) is charged to
// the enclosing category, so the categories' intervals never overlap and
// their sum never exceeds the solve.
int timer_begin(aerof_gpu_ctx* c, int cat) {
  Timers& t = c->timers;
  if (!t.on) return -1;
  if (t.depth > 0) {
    ++t.depth;
    return -2;
  }
  cudaEvent_t e[2];
  for (int k = 0; k < 2; ++k) {
    if (!t.pool.empty()) { e[k] = t.pool.back(); t.pool.pop_back(); }
    else AEROF_CUDA(cudaEventCreate(&e[k]));
  }
  AEROF_CUDA(cudaEventRecord(e[0], c->stream));
  t.recs.push_back({cat, e[0], e[1]});
  ++t.depth;
  return (int)t.recs.size() - 1;
}

void timer_end(aerof_gpu_ctx* c, int h) {
  if (h == -1) return;
  --c->timers.depth;
  if (h < 0) return;
  cudaEventRecord(c->timers.recs[h].b, c->stream);
}

static void timers_collect(aerof_gpu_ctx* c) {
  Timers& t = c->timers;
  if (t.recs.empty()) return;
  AEROF_CUDA(cudaStreamSynchronize(c->stream));
  for (auto& r : t.recs) {
    float ms = 0.f;
    AEROF_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
    t.ms[r.cat] += ms;
    t.cnt[r.cat] += 1;
    t.pool.push_back(r.a);
    t.pool.push_back(r.b);
  }
  t.recs.clear();
}

}  // namespace aerof

using namespace aerof;

extern "C" int aerof_gpu_profile(aerof_gpu_ctx* c, int enable) {
  return guard(c, [&]() -> int {
    if (!enable) timers_collect(c);
    c->timers.on = enable != 0;
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_timers(aerof_gpu_ctx* c, double* ms, long long* count, int n) {
  return guard(c, [&]() -> int {
    if (n < 0) return AEROF_EINVAL;
    timers_collect(c);
    for (int k = 0; k < AEROF_T_COUNT; ++k) {
      if (k < n) {
        if (ms) ms[k] = c->timers.ms[k];
        if (count) count[k] = c->timers.cnt[k];
      }
      c->timers.ms[k] = 0.0;
      c->timers.cnt[k] = 0;
    }
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_create(const aerof_gpu_config* cfg, aerof_gpu_ctx** out) {
  if (!cfg || !out) return AEROF_EINVAL;
  *out = nullptr;
  if (!(cfg->gamma > 1.0) || cfg->beta < 0.0 || cfg->beta > 0.5 ||
      (cfg->reconstruction != AEROF_REC_CONSTANT && cfg->reconstruction != AEROF_REC_VANALBADA &&
       cfg->reconstruction != AEROF_REC_LINEAR) ||
      (cfg->residual_kernel != AEROF_KERNEL_BLOCKED && cfg->residual_kernel != AEROF_KERNEL_EDGE))
    return AEROF_EINVAL;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) {
    cudaGetLastError();
    return AEROF_ECUDA;
  }
  aerof_gpu_ctx* c = new aerof_gpu_ctx();
  c->cfg = *cfg;
  c->dev = cfg->device;
  if (cudaSetDevice(c->dev) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return AEROF_ECUDA;
  }
  c->stream = c->own_stream;
  // loads the residual module and reserves the allocation-free scratch now,
  // before the caller can hand the rest of the device to its own pool
  noalloc_attach(c);
  *out = c;
  return AEROF_OK;
}

extern "C" int aerof_gpu_destroy(aerof_gpu_ctx* c) {
  if (!c) return AEROF_EINVAL;
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->stream);
  cudaStream_t own = c->own_stream;
  delete c;  // releases every device buffer
  if (own) cudaStreamDestroy(own);
  return AEROF_OK;
}

std::atomic<long long> aerof::g_launch_count{0};

extern "C" int aerof_gpu_launch_count(long long* count) {
  if (!count) return AEROF_EINVAL;
  *count = aerof::g_launch_count.exchange(0);
  return AEROF_OK;
}

extern "C" int aerof_gpu_set_stream(aerof_gpu_ctx* c, void* stream) {
  if (!c) return AEROF_EINVAL;
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return AEROF_OK;
}

extern "C" int aerof_gpu_last_error(aerof_gpu_ctx* c, char* buf, int len) {
  if (!c || !buf || len <= 0) return AEROF_EINVAL;
  std::strncpy(buf, c->last_error.c_str(), (size_t)len - 1);
  buf[len - 1] = 0;
  return AEROF_OK;
}
