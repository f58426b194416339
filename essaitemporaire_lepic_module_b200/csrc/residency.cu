// Device-resident mirrors of the Fortran host arrays for the drop-in
// routines.
//
// Without residency every drop-in copies its inputs to the GPU and its
// outputs back (the behaviour a Fortran caller gets by linking the library
// and changing nothing).  With residency on, each host array a drop-in
// touches gets one device mirror, keyed by its host byte range, created (and
// filled from the host) on first use and kept between calls.  Routines read
// and write the mirrors; the host copy goes stale until
// lepic_gpu_sync_to_host() / lepic_gpu_update_host() bring it back, which the
// caller does before host code reads the arrays (write_data and the backups
// at Src/main.f90:1294-1330).  Host code that writes an array the GPU holds
// says so with lepic_gpu_update_device(); the host-side loop statements of
// the timestep that touch mirrored arrays have device counterparts:
// lepic_gpu_mirror_zero for np(:,:,:,ptype,iproc) = 0 (Src/main.f90:1273)
// and lepic_gpu_mirror_copy for the one-rank MPI_ALLGATHERV of phi_dom into
// phi (Src/main.f90:977).
//
// Particle slices vxp(6, 1:nmax, ptype, iproc) are mirrored as SoA species
// (the layout of the kernels) with their flag_dead(1:nmax, ptype, iproc)
// slice; np_tot stays a host array that every call updates.  Particles
// appended on the host (part_injection and part_flux_injection write
// vxp(:, np_tot+1:) and raise np_tot, Src/injection.f90) are picked up by the
// next call: the host np_tot above the mirror's count means that the slots
// in between were written on the host and are uploaded.
//
// Mirrors never overlap.  A request that overlaps existing mirrors without
// lying inside one of them retires them (downloading device-newer ones first)
// and creates one mirror over the union of the ranges.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

#include "lepic_internal.cuh"

namespace lepic {

__global__ void k_aos_to_soa_range(const double *aos, double *soa, long long first, long long n,
                                   long long cap) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 6 * n) return;
  long long i = t / 6;
  int c = (int)(t % 6);
  soa[c * cap + first + i] = aos[t];
}

__global__ void k_soa_to_aos_range(const double *soa, double *aos, long long n, long long cap) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 6 * n) return;
  long long i = t / 6;
  int c = (int)(t % 6);
  aos[t] = soa[c * cap + i];
}

int aos_to_soa(const double *aos, double *soa, long long first, long long n, long long cap, cudaStream_t s) {
  if (n <= 0) return LEPIC_OK;
  k_aos_to_soa_range<<<grid_for(6 * n, 256), 256, 0, s>>>(aos, soa, first, n, cap);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int soa_to_aos(const double *soa, double *aos, long long n, long long cap, cudaStream_t s) {
  if (n <= 0) return LEPIC_OK;
  k_soa_to_aos_range<<<grid_for(6 * n, 256), 256, 0, s>>>(soa, aos, n, cap);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

namespace {

std::recursive_mutex g_mu;
bool g_on = false;
long long g_h2d = 0, g_d2h = 0;
unsigned long long g_gen = 0;

struct Mirror {
  uintptr_t h0 = 0, h1 = 0;  // host byte range [h0, h1)
  char *dev = nullptr;       // plain mirror: device copy of the range
  bool newer = false;        // the device holds writes the host has not seen
  unsigned long long gen = 0;  // changes whenever the host content is (re)loaded
  // particle slice vxp(6, 1:nmax): SoA species on the device
  bool particles = false;
  lepic_species_f64_t sp{};
  int n = 0;                    // particle count of the mirror (host view)
  signed char *fd_h = nullptr;  // host flag_dead slice of the species
  bool fd_newer = false;
};

std::map<uintptr_t, Mirror> g_mir;  // by h0

int h2d(void *d, const void *h, size_t bytes, cudaStream_t s) {
  if (!bytes) return LEPIC_OK;
  LEPIC_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s));
  g_h2d += (long long)bytes;
  return LEPIC_OK;
}

int d2h(void *h, const void *d, size_t bytes, cudaStream_t s) {
  if (!bytes) return LEPIC_OK;
  LEPIC_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s));
  g_d2h += (long long)bytes;
  return LEPIC_OK;
}

void free_mirror(Mirror &m) {
  if (m.particles) {
    cudaFree(m.sp.p);
    cudaFree(m.sp.p_alt);
    cudaFree(m.sp.key);
    cudaFree(m.sp.count);
    cudaFree(m.sp.flag_dead);
  } else {
    cudaFree(m.dev);
  }
  m = Mirror();
}

// Bring the host copy of m up to date.
int download(Mirror &m, cudaStream_t s) {
  if (m.particles) {
    if (m.newer && m.n > 0) {
      double *aos = (double *)scratch("mirror_aos", sizeof(double) * 6 * (size_t)m.n);
      if (!aos) return LEPIC_ERR_CUDA;
      int rc = soa_to_aos(m.sp.p, aos, m.n, m.sp.cap, s);
      if (rc) return rc;
      rc = d2h((void *)m.h0, aos, sizeof(double) * 6 * (size_t)m.n, s);
      if (rc) return rc;
    }
    if (m.fd_newer && m.fd_h) {
      int rc = d2h(m.fd_h, m.sp.flag_dead, (size_t)m.sp.cap, s);
      if (rc) return rc;
    }
    LEPIC_CUDA(cudaStreamSynchronize(s));
    m.newer = m.fd_newer = false;
    return LEPIC_OK;
  }
  if (!m.newer) return LEPIC_OK;
  int rc = d2h((void *)m.h0, m.dev, m.h1 - m.h0, s);
  if (rc) return rc;
  LEPIC_CUDA(cudaStreamSynchronize(s));
  m.newer = false;
  return LEPIC_OK;
}

// The mirror that contains [a, b), or null.
Mirror *containing(uintptr_t a, uintptr_t b) {
  auto it = g_mir.upper_bound(a);
  if (it == g_mir.begin()) return nullptr;
  --it;
  Mirror &m = it->second;
  return (m.h0 <= a && b <= m.h1) ? &m : nullptr;
}

// Retire every mirror overlapping [a, b) after bringing the host up to date;
// widens [a, b) to the union when `widen`.
int retire_overlapping(uintptr_t &a, uintptr_t &b, bool widen, bool keep_host, cudaStream_t s) {
  auto it = g_mir.upper_bound(a);
  if (it != g_mir.begin()) --it;
  while (it != g_mir.end() && it->second.h0 < b) {
    Mirror &m = it->second;
    if (m.h1 <= a) {
      ++it;
      continue;
    }
    if (keep_host) {
      int rc = download(m, s);
      if (rc) return rc;
    }
    if (widen && !m.particles) {
      a = std::min(a, m.h0);
      b = std::max(b, m.h1);
    }
    free_mirror(m);
    it = g_mir.erase(it);
  }
  return LEPIC_OK;
}

Mirror *new_plain(uintptr_t a, uintptr_t b, cudaStream_t s, int *rc) {
  Mirror m;
  m.h0 = a;
  m.h1 = b;
  if (cudaMalloc(&m.dev, b - a) != cudaSuccess) {
    *rc = LEPIC_ERR_CUDA;
    return nullptr;
  }
  *rc = h2d(m.dev, (const void *)a, b - a, s);
  if (*rc) {
    cudaFree(m.dev);
    return nullptr;
  }
  m.gen = ++g_gen;
  return &(g_mir[a] = m);
}

}  // namespace

bool residency_on() {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return g_on;
}

void *mirror_array(const void *h, size_t bytes, bool write, cudaStream_t s, int *rc) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  *rc = LEPIC_OK;
  uintptr_t a = (uintptr_t)h, b = a + (bytes ? bytes : 1);
  Mirror *m = containing(a, b);
  if (m && m->particles) m = nullptr;
  if (!m) {
    *rc = retire_overlapping(a, b, true, true, s);
    if (*rc) return nullptr;
    m = new_plain(a, b, s, rc);
    if (!m) return nullptr;
  }
  if (write) m->newer = true;
  return m->dev + ((uintptr_t)h - m->h0);
}

unsigned long long mirror_generation(const void *h) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  uintptr_t a = (uintptr_t)h;
  Mirror *m = containing(a, a + 1);
  return m ? m->gen : 0;
}

int mirror_to_host(const void *h, size_t bytes, cudaStream_t s) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  uintptr_t a = (uintptr_t)h, b = a + bytes;
  auto it = g_mir.upper_bound(a);
  if (it != g_mir.begin()) --it;
  for (; it != g_mir.end() && it->second.h0 < b; ++it) {
    if (it->second.h1 <= a) continue;
    int rc = download(it->second, s);
    if (rc) return rc;
  }
  return LEPIC_OK;
}

int mirror_species(double *vxp_h, int np_h, int nmax, signed char *fd_h, cudaStream_t s,
                   lepic_species_f64_t *out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (nmax < 1 || np_h < 0 || np_h > nmax) return LEPIC_ERR_ARG;
  uintptr_t a = (uintptr_t)vxp_h, b = a + sizeof(double) * 6 * (size_t)nmax;
  Mirror *m = containing(a, b);
  if (m && !(m->particles && m->h0 == a && m->h1 == b)) m = nullptr;
  const long long cap = nmax;
  if (!m) {
    int rc = retire_overlapping(a, b, false, true, s);
    if (rc) return rc;
    Mirror nm;
    nm.h0 = a;
    nm.h1 = b;
    nm.particles = true;
    nm.sp.cap = nmax;
    bool ok = cudaMalloc(&nm.sp.p, sizeof(double) * 6 * cap) == cudaSuccess &&
              cudaMalloc(&nm.sp.p_alt, sizeof(double) * 6 * cap) == cudaSuccess &&
              cudaMalloc(&nm.sp.key, sizeof(int) * cap) == cudaSuccess &&
              cudaMalloc(&nm.sp.count, sizeof(int)) == cudaSuccess &&
              cudaMalloc(&nm.sp.flag_dead, (size_t)cap) == cudaSuccess;
    if (!ok) {
      free_mirror(nm);
      return LEPIC_ERR_CUDA;
    }
    LEPIC_CUDA(cudaMemsetAsync(nm.sp.flag_dead, 0, (size_t)cap, s));
    if (fd_h) {
      rc = h2d(nm.sp.flag_dead, fd_h, (size_t)cap, s);
      if (rc) return rc;
      nm.fd_h = fd_h;
    }
    nm.n = 0;
    nm.gen = ++g_gen;
    m = &(g_mir[a] = nm);
  } else if (fd_h && m->fd_h != fd_h) {
    // first call that names the flag_dead slice: the host copy is current
    int rc = h2d(m->sp.flag_dead, fd_h, (size_t)cap, s);
    if (rc) return rc;
    m->fd_h = fd_h;
    m->fd_newer = false;
  }
  if (np_h < m->n) {
    fprintf(stderr,
            "lepic_gpu: np_tot (%d) below the %d particles of the device mirror; the host must "
            "call lepic_gpu_update_device after changing a mirrored particle array\n",
            np_h, m->n);
    return LEPIC_ERR_ARG;
  }
  if (np_h > m->n) {
    // slots m->n .. np_h-1 were written on the host (injection, first use)
    long long k = np_h - m->n;
    double *aos = (double *)scratch("mirror_aos", sizeof(double) * 6 * (size_t)k);
    if (!aos) return LEPIC_ERR_CUDA;
    int rc = h2d(aos, vxp_h + 6LL * m->n, sizeof(double) * 6 * (size_t)k, s);
    if (rc) return rc;
    rc = aos_to_soa(aos, m->sp.p, m->n, k, cap, s);
    if (rc) return rc;
    if (m->fd_h) {
      rc = h2d(m->sp.flag_dead + m->n, m->fd_h + m->n, (size_t)k, s);
      if (rc) return rc;
    }
    m->n = np_h;
  }
  int rc = h2d(m->sp.count, &m->n, sizeof(int), s);
  if (rc) return rc;
  LEPIC_CUDA(cudaStreamSynchronize(s));  // m->n is read by the copy above
  *out = m->sp;
  return LEPIC_OK;
}

int mirror_species_done(double *vxp_h, const lepic_species_f64_t &sp, bool wrote, bool fd_wrote,
                        int *np_out, cudaStream_t s) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  uintptr_t a = (uintptr_t)vxp_h;
  Mirror *m = containing(a, a + 1);
  if (!m || !m->particles) return LEPIC_ERR_ARG;
  m->sp = sp;  // the sort swaps the two particle buffers
  int n = 0;
  int rc = d2h(&n, sp.count, sizeof(int), s);
  if (rc) return rc;
  LEPIC_CUDA(cudaStreamSynchronize(s));
  if (n > sp.cap) n = sp.cap;
  m->n = n;
  if (wrote) m->newer = true;
  if (fd_wrote) m->fd_newer = true;
  if (np_out) *np_out = n;
  return LEPIC_OK;
}

int mirror_h2d(void *d, const void *h, size_t bytes, cudaStream_t s) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return h2d(d, h, bytes, s);
}

int mirror_d2h(void *h, const void *d, size_t bytes, cudaStream_t s) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return d2h(h, d, bytes, s);
}

}  // namespace lepic

using namespace lepic;

extern "C" {

int lepic_gpu_set_residency(int on) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!on && g_on) {
    int rc = lepic_gpu_release_all();
    if (rc) return rc;
  }
  g_on = on != 0;
  return LEPIC_OK;
}

int lepic_gpu_residency(void) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  return g_on ? 1 : 0;
}

int lepic_gpu_sync_to_host(void) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  for (auto &kv : g_mir) {
    int rc = download(kv.second, 0);
    if (rc) return rc;
  }
  return LEPIC_OK;
}

int lepic_gpu_update_host(const void *h, size_t bytes) {
  if (!h) return LEPIC_ERR_ARG;
  return mirror_to_host(h, bytes, 0);
}

int lepic_gpu_update_device(const void *h, size_t bytes) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!h) return LEPIC_ERR_ARG;
  uintptr_t a = (uintptr_t)h, b = a + bytes;
  auto it = g_mir.upper_bound(a);
  if (it != g_mir.begin()) --it;
  while (it != g_mir.end() && it->second.h0 < b) {
    Mirror &m = it->second;
    if (m.h1 <= a) {
      ++it;
      continue;
    }
    if (m.particles) {
      // the host rewrote particles: the next call reloads the slice
      free_mirror(m);
      it = g_mir.erase(it);
      continue;
    }
    uintptr_t lo = std::max(a, m.h0), hi = std::min(b, m.h1);
    int rc = h2d(m.dev + (lo - m.h0), (const void *)lo, hi - lo, 0);
    if (rc) return rc;
    m.gen = ++g_gen;
    ++it;
  }
  LEPIC_CUDA(cudaStreamSynchronize(0));
  return LEPIC_OK;
}

int lepic_gpu_release(const void *h, size_t bytes) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!h) return LEPIC_ERR_ARG;
  uintptr_t a = (uintptr_t)h, b = a + bytes;
  return retire_overlapping(a, b, false, true, 0);
}

int lepic_gpu_release_all(void) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  int rc = lepic_gpu_sync_to_host();
  for (auto &kv : g_mir) free_mirror(kv.second);
  g_mir.clear();
  return rc;
}

int lepic_gpu_mirror_zero(void *h, size_t bytes) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!h) return LEPIC_ERR_ARG;
  if (!g_on) {
    memset(h, 0, bytes);
    return LEPIC_OK;
  }
  int rc = LEPIC_OK;
  void *d = mirror_array(h, bytes, true, 0, &rc);
  if (!d) return rc ? rc : LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemsetAsync(d, 0, bytes, 0));
  return LEPIC_OK;
}

int lepic_gpu_mirror_copy(void *dst, const void *src, size_t bytes) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!dst || !src) return LEPIC_ERR_ARG;
  uintptr_t d0 = (uintptr_t)dst, s0 = (uintptr_t)src;
  if (d0 < s0 + bytes && s0 < d0 + bytes) return LEPIC_ERR_ARG;
  if (!g_on) {
    memcpy(dst, src, bytes);
    return LEPIC_OK;
  }
  int rc = LEPIC_OK;
  void *dd = mirror_array(dst, bytes, true, 0, &rc);
  if (!dd) return rc ? rc : LEPIC_ERR_CUDA;
  const void *sd = mirror_array(src, bytes, false, 0, &rc);
  if (!sd) return rc ? rc : LEPIC_ERR_CUDA;
  // the source lookup may have merged the destination's mirror into a wider
  // one; the destination range now lies inside a mirror, so this lookup
  // only finds it
  dd = mirror_array(dst, bytes, true, 0, &rc);
  if (!dd) return rc ? rc : LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemcpyAsync(dd, sd, bytes, cudaMemcpyDeviceToDevice, 0));
  return LEPIC_OK;
}

int lepic_gpu_mirror_stats(long long *h2d_bytes, long long *d2h_bytes, int *mirrors) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (h2d_bytes) *h2d_bytes = g_h2d;
  if (d2h_bytes) *d2h_bytes = g_d2h;
  if (mirrors) *mirrors = (int)g_mir.size();
  return LEPIC_OK;
}

}  // extern "C"
