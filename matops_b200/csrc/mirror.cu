// Device mirrors of host backing arrays (mo_mirror_*): the residency layer a Go shim needs
// to keep FloatMatrix data on the GPU across a chain of calls.
//
// The reference operates in place on views of host slices (FloatArray() + LeadingIndex(),
// mmult.go:228-233); views of one backing array overlap freely (partition.go:210-340).  A
// mirror covers one whole registered array [host, host + count): every view inside it maps
// to the same device memory at the same element offset, so overlapping views see each
// other's results without host round trips.  Coherence is per mirror, in three states:
//   kSync        host and device copies are equal
//   kHostNewer   the caller changed the host copy (mo_mirror_host_modified, or just
//                registered): the next device view uploads the whole array first
//   kDeviceNewer a device view was taken for writing: mo_mirror_to_host downloads
// Lookups go by address: mo_mirror_find returns the registered array that contains a host
// pointer and the pointer's element offset, which is how a shim maps an arbitrary view
// (whose FloatArray() starts inside the root array) to its mirror.
#include <map>
#include <mutex>

#include "context.cuh"

struct mo_mirror {
  mo_ctx *ctx = nullptr;
  double *host = nullptr;
  int64_t count = 0;
  double *dev = nullptr;
  int state = 0;
};

namespace {

enum { kSync = 0, kHostNewer = 1, kDeviceNewer = 2 };

// registry: host base address -> mirror, per process (mirrors carry their context)
std::mutex g_mu;
std::map<uintptr_t, mo_mirror *> g_mirrors;

uintptr_t addr(const void *p) { return reinterpret_cast<uintptr_t>(p); }

// the mirror whose range contains p (registry lock held)
mo_mirror *containing(const void *p) {
  auto it = g_mirrors.upper_bound(addr(p));
  if (it == g_mirrors.begin()) return nullptr;
  --it;
  mo_mirror *m = it->second;
  return addr(p) < addr(m->host + m->count) ? m : nullptr;
}

int ensure_device(mo_mirror *m) {
  if (!m->dev) {
    MO_CUDA_TRY(cudaMalloc(&m->dev, (size_t)m->count * sizeof(double)));
    m->state = kHostNewer;
  }
  if (m->state == kHostNewer) {
    MO_CUDA_TRY(cudaMemcpyAsync(m->dev, m->host, (size_t)m->count * sizeof(double),
                                cudaMemcpyHostToDevice, m->ctx->stream));
    m->state = kSync;
  }
  return MO_OK;
}

}  // namespace

extern "C" {

int mo_mirror_create(mo_ctx *ctx, double *host, int64_t count, mo_mirror **out) {
  if (!ctx || !host || count <= 0 || !out) return MO_EINVAL;
  std::lock_guard<std::mutex> lock(g_mu);
  // a range that overlaps a registered one is refused: views of a registered array are
  // found with mo_mirror_find instead
  mo_mirror *a = containing(host), *b = containing(host + count - 1);
  auto nx = g_mirrors.lower_bound(addr(host));
  if (a || b || (nx != g_mirrors.end() && nx->first < addr(host + count))) return MO_EINVAL;
  mo_mirror *m = new mo_mirror();
  m->ctx = ctx;
  m->host = host;
  m->count = count;
  m->state = kHostNewer;
  g_mirrors[addr(host)] = m;
  *out = m;
  return MO_OK;
}

int mo_mirror_destroy(mo_mirror *m) {
  if (!m) return MO_EINVAL;
  std::lock_guard<std::mutex> lock(g_mu);
  g_mirrors.erase(addr(m->host));
  int rc = MO_OK;
  if (m->dev) {
    if (cudaSetDevice(m->ctx->device) != cudaSuccess ||
        cudaStreamSynchronize(m->ctx->stream) != cudaSuccess || cudaFree(m->dev) != cudaSuccess)
      rc = MO_ECUDA;
  }
  delete m;
  return rc;
}

int mo_mirror_find(const double *p, mo_mirror **m, int64_t *offset) {
  if (!p || !m) return MO_EINVAL;
  std::lock_guard<std::mutex> lock(g_mu);
  mo_mirror *c = containing(p);
  *m = c;
  if (!c) return MO_EINVAL;
  if (offset) *offset = (int64_t)(p - c->host);
  return MO_OK;
}

int mo_mirror_view(mo_mirror *m, const double *p, int64_t rows, int64_t cols, int64_t ld,
                   int write, mo_matrix *out) {
  if (!m || !p || !out || rows < 0 || cols < 0) return MO_EINVAL;
  const int64_t off = (int64_t)(p - m->host);
  if (p < m->host || off >= m->count) return MO_EINVAL;
  if (rows > 0 && cols > 0) {
    if (ld < rows) return MO_EINVAL;
    const int64_t last = off + (rows - 1) + (cols - 1) * ld;  // the view's last element
    if (last >= m->count) return MO_EINVAL;
  }
  int rc = mo::enter(m->ctx);
  if (rc) return rc;
  std::lock_guard<std::mutex> lock(g_mu);
  if ((rc = ensure_device(m))) return rc;
  if (write) m->state = kDeviceNewer;
  out->data = m->dev + off;
  out->rows = rows;
  out->cols = cols;
  out->ld = ld < 1 ? 1 : ld;
  return MO_OK;
}

int mo_mirror_to_host(mo_mirror *m) {
  if (!m) return MO_EINVAL;
  int rc = mo::enter(m->ctx);
  if (rc) return rc;
  std::lock_guard<std::mutex> lock(g_mu);
  if (m->state == kDeviceNewer) {
    MO_CUDA_TRY(cudaMemcpyAsync(m->host, m->dev, (size_t)m->count * sizeof(double),
                                cudaMemcpyDeviceToHost, m->ctx->stream));
    m->state = kSync;
  }
  MO_CUDA_TRY(cudaStreamSynchronize(m->ctx->stream));
  return MO_OK;
}

int mo_mirror_host_modified(mo_mirror *m) {
  if (!m) return MO_EINVAL;
  std::lock_guard<std::mutex> lock(g_mu);
  if (m->state == kDeviceNewer) return MO_EINVAL;  // both copies changed: refuse to guess
  m->state = kHostNewer;
  return MO_OK;
}

int mo_mirror_state(const mo_mirror *m) { return m ? m->state : MO_EINVAL; }

}  // extern "C"
