// hb_api.cu -- C ABI of the B200-native force-and-constraint path: object
// lifetimes, validation with the reference's error semantics, and the
// per-step orchestration (integrator sub-steps, constraint hooks, device-
// gated neighbour rebuild, pair kernel overlapped with SPME on a second
// stream, force combine).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>
#include <vector>

#include "hb_internal.cuh"

static thread_local std::string g_err;
static std::atomic<uint64_t> g_uid{1};
uint64_t hb_next_uid() { return g_uid.fetch_add(1); }

void hb_set_error(const std::string &msg) { g_err = msg; }
int hb_fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

extern "C" const char *hb_last_error(void) { return g_err.c_str(); }
extern "C" const char *hb_version(void) { return "heddle_b200 0.1 (sm_100a)"; }


// ---------------------------------------------------------------------
// context
// ---------------------------------------------------------------------
extern "C" int hb_context_create(int device_ordinal, hb_context **out) {
  HB_REQUIRE(out != nullptr, HB_ERR_INVALID_ARGUMENT, "out is null");
  int count = 0;
  HB_CUDA(cudaGetDeviceCount(&count));
  HB_REQUIRE(device_ordinal >= 0 && device_ordinal < count, HB_ERR_INVALID_ARGUMENT,
             "device ordinal out of range");
  HB_CUDA(cudaSetDevice(device_ordinal));
  hb_context *c = new hb_context();
  c->device = device_ordinal;
  cudaDeviceProp prop;
  HB_CUDA(cudaGetDeviceProperties(&prop, device_ordinal));
  if (prop.major < 10) {
    delete c;
    return hb_fail(HB_ERR_UNSUPPORTED, "heddle_b200 is built for sm_100a (B200)");
  }
  c->n_sm = prop.multiProcessorCount;
  HB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  // the reciprocal-space chain is the step's critical path: its stream gets
  // the highest priority, so its blocks go first whenever SM room frees up
  int prio_lo = 0, prio_hi = 0;
  HB_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  HB_CUDA(cudaStreamCreateWithPriority(&c->stream2, cudaStreamNonBlocking, prio_hi));
  HB_CUDA(cudaStreamCreateWithFlags(&c->stream3, cudaStreamNonBlocking));
  HB_CUDA(cudaStreamCreateWithFlags(&c->stream4, cudaStreamNonBlocking));
  HB_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  HB_CUDA(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
  HB_CUDA(cudaEventCreateWithFlags(&c->ev_xfork, cudaEventDisableTiming));
  HB_CUDA(cudaEventCreateWithFlags(&c->ev_xjoin, cudaEventDisableTiming));
  *out = c;
  return HB_OK;
}

extern "C" int hb_context_destroy(hb_context *ctx) {
  if (!ctx) return HB_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStreamSynchronize(ctx->stream2);
  for (auto e : ctx->tev) cudaEventDestroy(e);
  cudaEventDestroy(ctx->ev_fork);
  cudaEventDestroy(ctx->ev_join);
  cudaEventDestroy(ctx->ev_xfork);
  cudaEventDestroy(ctx->ev_xjoin);
  cudaStreamDestroy(ctx->stream);
  cudaStreamDestroy(ctx->stream2);
  cudaStreamDestroy(ctx->stream3);
  cudaStreamDestroy(ctx->stream4);
  delete ctx;
  return HB_OK;
}

extern "C" int hb_context_synchronize(hb_context *ctx) {
  HB_REQUIRE(ctx, HB_ERR_INVALID_ARGUMENT, "null context");
  HB_CUDA(cudaStreamSynchronize(ctx->stream));
  HB_CUDA(cudaStreamSynchronize(ctx->stream2));
  return HB_OK;
}

// ---------------------------------------------------------------------
// timing: event pairs per stage, summed at the end of a call
// ---------------------------------------------------------------------
struct StageTimer {
  hb_context *ctx;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
  size_t used = 0;
  cudaEvent_t get() {
    if (used < ctx->tev.size()) return ctx->tev[used++];
    cudaEvent_t e;
    cudaEventCreate(&e);
    ctx->tev.push_back(e);
    used++;
    return e;
  }
};
static thread_local StageTimer *g_timer = nullptr;

static cudaEvent_t stage_begin(cudaStream_t s) {
  if (!g_timer) return nullptr;
  cudaEvent_t e = g_timer->get();
  cudaEventRecord(e, s);
  return e;
}
static void stage_end(int stage, cudaEvent_t b, cudaStream_t s) {
  if (!g_timer || !b) return;
  cudaEvent_t e = g_timer->get();
  cudaEventRecord(e, s);
  g_timer->marks.push_back({stage, {b, e}});
}

// ---------------------------------------------------------------------
// system
// ---------------------------------------------------------------------
static DBox make_dbox(const double b[6]) { return hb_make_dbox(b); }

static bool finite6(const double b[6]) {
  for (int d = 0; d < 6; ++d)
    if (!std::isfinite(b[d])) return false;
  return b[0] > 0.0 && b[1] > 0.0 && b[2] > 0.0;
}

static void perp_widths(const double b[6], double w[3]) { hb_perp_widths(b, w); }

// wrap a position into the primary cell in FP64 (kernels/pbc.cuh:73-91)
static void wrap_host(const double b[6], double &x, double &y, double &z, int &ka, int &kb,
                      int &kc) {
  double sc = z / b[2];
  double sb = (y - sc * b[5]) / b[1];
  double sa = (x - sb * b[3] - sc * b[4]) / b[0];
  double fa = std::floor(sa + 0.5), fb = std::floor(sb + 0.5), fc = std::floor(sc + 0.5);
  x -= fa * b[0] + fb * b[3] + fc * b[4];
  y -= fb * b[1] + fc * b[5];
  z -= fc * b[2];
  ka = (int)fa;
  kb = (int)fb;
  kc = (int)fc;
}

// The FP64 lattice lives on the device (a barostat move changes it there);
// host code that needs the box reads it back first.
int sys_refresh_box(hb_system *sys) {
  HB_CUDA(cudaStreamSynchronize(sys->ctx->stream));
  HB_CUDA(cudaMemcpy(sys->box, sys->d_box64, sizeof(double) * 6, cudaMemcpyDeviceToHost));
  return HB_OK;
}

static int upload_state(hb_system *sys, const double *pos, const double *vel,
                        const int32_t *images_in, bool keep_images) {
  const uint32_t n = sys->n;
  sys->fix_valid = false;
  if (keep_images) HB_TRY(sys_refresh_box(sys));
  std::vector<float4> posq(n), v(n);
  std::vector<int4> img(n);
  std::vector<int4> old_img;
  if (keep_images && n) {
    old_img.resize(n);
    HB_CUDA(cudaMemcpy(old_img.data(), sys->d_image, sizeof(int4) * n, cudaMemcpyDeviceToHost));
  }
  for (uint32_t i = 0; i < n; ++i) {
    double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z))
      return hb_fail(HB_ERR_NOT_FINITE, "non-finite position for atom " + std::to_string(i));
    int ka, kb, kc;
    wrap_host(sys->box, x, y, z, ka, kb, kc);
    posq[i] = make_float4((float)x, (float)y, (float)z, (float)sys->h_charge[i]);
    int4 im;
    if (keep_images) {
      im = old_img[i];
      im.x += ka;
      im.y += kb;
      im.z += kc;
    } else {
      im.x = ka + (images_in ? images_in[3 * i] : 0);
      im.y = kb + (images_in ? images_in[3 * i + 1] : 0);
      im.z = kc + (images_in ? images_in[3 * i + 2] : 0);
    }
    im.w = (int)sys->h_type[i];
    img[i] = im;
    const double m = sys->h_mass[i];
    v[i] = make_float4(vel ? (float)vel[3 * i] : 0.f, vel ? (float)vel[3 * i + 1] : 0.f,
                       vel ? (float)vel[3 * i + 2] : 0.f, (float)(1.0 / m));
  }
  if (n) {
    HB_CUDA(cudaMemcpy(sys->d_posq, posq.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    HB_CUDA(cudaMemcpy(sys->d_image, img.data(), sizeof(int4) * n, cudaMemcpyHostToDevice));
    if (vel || !keep_images)
      HB_CUDA(cudaMemcpy(sys->d_vel, v.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    // the pre-drift snapshot is the constraints' reference frame: only a
    // new system initialises it
    if (!keep_images)
      HB_CUDA(cudaMemcpy(sys->d_pos_prev, posq.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
  }
  return HB_OK;
}

extern "C" int hb_system_create(hb_context *ctx, const hb_system_desc *d, hb_system **out) {
  HB_REQUIRE(ctx && d && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_REQUIRE(finite6(d->box), HB_ERR_NOT_FINITE, "box must be finite with positive diagonal");
  const uint32_t n = d->n_atoms;
  HB_REQUIRE(n == 0 || (d->positions && d->masses && d->charges && d->types),
             HB_ERR_INVALID_ARGUMENT, "positions, masses, charges and types are required");
  for (uint32_t i = 0; i < n; ++i) {
    HB_REQUIRE(std::isfinite(d->masses[i]) && d->masses[i] > 0.0, HB_ERR_INVALID_ARGUMENT,
               "masses must be finite and positive");
    HB_REQUIRE(std::isfinite(d->charges[i]), HB_ERR_NOT_FINITE, "charges must be finite");
  }
  HB_CUDA(cudaSetDevice(ctx->device));
  hb_system *s = new hb_system();
  s->ctx = ctx;
  s->n = n;
  std::memcpy(s->box, d->box, sizeof(double) * 6);
  s->h_mass.assign(d->masses, d->masses + n);
  s->h_charge.assign(d->charges, d->charges + n);
  s->h_type.assign(d->types, d->types + n);
  const size_t nn = std::max<size_t>(n, 1);
  HB_CUDA(cudaMalloc(&s->d_box, sizeof(DBox)));
  DBox db = make_dbox(d->box);
  HB_CUDA(cudaMemcpy(s->d_box, &db, sizeof(DBox), cudaMemcpyHostToDevice));
  HB_CUDA(cudaMalloc(&s->d_box64, sizeof(double) * 6));
  HB_CUDA(cudaMemcpy(s->d_box64, d->box, sizeof(double) * 6, cudaMemcpyHostToDevice));
  HB_CUDA(cudaMalloc(&s->d_posq, sizeof(float4) * nn));
  HB_CUDA(cudaMalloc(&s->d_vel, sizeof(float4) * nn));
  HB_CUDA(cudaMalloc(&s->d_image, sizeof(int4) * nn));
  HB_CUDA(cudaMalloc(&s->d_force, sizeof(float4) * nn));
  HB_CUDA(cudaMemset(s->d_force, 0, sizeof(float4) * nn));
  HB_CUDA(cudaMalloc(&s->d_pos_prev, sizeof(float4) * nn));
  HB_CUDA(cudaMalloc(&s->d_vfix, sizeof(long long) * 3 * nn));
  HB_CUDA(cudaMemset(s->d_vfix, 0, sizeof(long long) * 3 * nn));
  HB_CUDA(cudaMalloc(&s->d_xfix, sizeof(long long) * 3 * nn));
  HB_CUDA(cudaMemset(s->d_xfix, 0, sizeof(long long) * 3 * nn));
  HB_CUDA(cudaMalloc(&s->d_red, sizeof(double) * (4 * 296 + 8)));
  HB_CUDA(cudaMallocHost(&s->h_red, sizeof(double) * 8));
  int rc = upload_state(s, d->positions, d->velocities, d->images, false);
  if (rc != HB_OK) {
    hb_system_destroy(s);
    return rc;
  }
  *out = s;
  return HB_OK;
}

extern "C" int hb_system_destroy(hb_system *s) {
  if (!s) return HB_OK;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  cudaFree(s->d_box);
  cudaFree(s->d_box64);
  cudaFree(s->d_posq);
  cudaFree(s->d_vel);
  cudaFree(s->d_image);
  cudaFree(s->d_force);
  cudaFree(s->d_pos_prev);
  cudaFree(s->d_vfix);
  cudaFree(s->d_xfix);
  cudaFree(s->d_red);
  cudaFreeHost(s->h_red);
  cudaFree(s->d_stage);
  cudaFree(s->d_stage_img);
  cudaFree(s->d_bad);
  delete s;
  return HB_OK;
}

// ---- state transfer: FP64 host arrays <-> the device SoA, converted on the
// device (the host only copies), so a per-step exchange costs the PCIe
// transfers and two small kernels.
namespace {

template <class T>
__global__ void k_state_check(const T *__restrict__ pos, uint32_t *__restrict__ bad, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!isfinite(pos[3 * i]) || !isfinite(pos[3 * i + 1]) || !isfinite(pos[3 * i + 2]))
    atomicMin(bad, i);
}

// wrap into the primary cell in FP64, operation by operation as the host
// upload does it (no contraction), keeping image counts continuous.  With a
// `bad` word (set by k_state_check earlier on the same stream) nothing is
// written when some position is not finite, so the state is left as it was
template <class T>
__global__ void k_state_in(const T *__restrict__ pos, const T *__restrict__ vel,
                           const double *__restrict__ b, float4 *__restrict__ posq,
                           float4 *__restrict__ v, int4 *__restrict__ image,
                           const uint32_t *__restrict__ bad, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (bad && *bad != 0xFFFFFFFFu) return;
  if (pos) {
    double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    const double sc = __ddiv_rn(z, b[2]);
    const double sb = __ddiv_rn(__dsub_rn(y, __dmul_rn(sc, b[5])), b[1]);
    const double sa =
        __ddiv_rn(__dsub_rn(__dsub_rn(x, __dmul_rn(sb, b[3])), __dmul_rn(sc, b[4])), b[0]);
    const double fa = floor(__dadd_rn(sa, 0.5)), fb = floor(__dadd_rn(sb, 0.5)),
                 fc = floor(__dadd_rn(sc, 0.5));
    x = __dsub_rn(x, __dadd_rn(__dadd_rn(__dmul_rn(fa, b[0]), __dmul_rn(fb, b[3])),
                               __dmul_rn(fc, b[4])));
    y = __dsub_rn(y, __dadd_rn(__dmul_rn(fb, b[1]), __dmul_rn(fc, b[5])));
    z = __dsub_rn(z, __dmul_rn(fc, b[2]));
    float4 p = posq[i];
    p.x = (float)x;
    p.y = (float)y;
    p.z = (float)z;
    posq[i] = p;
    int4 im = image[i];
    im.x += (int)fa;
    im.y += (int)fb;
    im.z += (int)fc;
    image[i] = im;
  }
  if (vel) {
    float4 q = v[i];
    q.x = (float)vel[3 * i];
    q.y = (float)vel[3 * i + 1];
    q.z = (float)vel[3 * i + 2];
    v[i] = q;
  }
}

template <class T>
__global__ void k_state_out(const float4 *__restrict__ posq, const float4 *__restrict__ vel,
                            const float4 *__restrict__ force, const int4 *__restrict__ image,
                            T *__restrict__ pos, T *__restrict__ velo, T *__restrict__ frc,
                            int32_t *__restrict__ img, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (pos) {
    const float4 p = posq[i];
    pos[3 * i] = p.x;
    pos[3 * i + 1] = p.y;
    pos[3 * i + 2] = p.z;
  }
  if (velo) {
    const float4 q = vel[i];
    velo[3 * i] = q.x;
    velo[3 * i + 1] = q.y;
    velo[3 * i + 2] = q.z;
  }
  if (frc) {
    const float4 f = force[i];
    frc[3 * i] = f.x;
    frc[3 * i + 1] = f.y;
    frc[3 * i + 2] = f.z;
  }
  if (img) {
    const int4 m = image[i];
    img[3 * i] = m.x;
    img[3 * i + 1] = m.y;
    img[3 * i + 2] = m.z;
  }
}

int stage_alloc(hb_system *sys) {
  if (sys->d_stage) return HB_OK;
  const size_t nn = std::max<size_t>(sys->n, 1);
  HB_CUDA(cudaMalloc(&sys->d_stage, sizeof(double) * 9 * nn));
  HB_CUDA(cudaMalloc(&sys->d_stage_img, sizeof(int32_t) * 3 * nn));
  HB_CUDA(cudaMalloc(&sys->d_bad, sizeof(uint32_t)));
  return HB_OK;
}

}  // namespace

namespace {

// Upload: both host arrays and the finite check are queued before the one
// synchronisation; the conversion writes nothing when a position is not
// finite (checked on the device), so a rejected call leaves the state as it
// was.  T is the host element type (double or float).
template <class T>
int set_state_t(hb_system *sys, const T *positions, const T *velocities) {
  HB_REQUIRE(sys, HB_ERR_INVALID_ARGUMENT, "null system");
  const uint32_t n = sys->n;
  if (!n || (!positions && !velocities)) return HB_OK;
  HB_TRY(stage_alloc(sys));
  cudaStream_t s = sys->ctx->stream;
  T *dp = reinterpret_cast<T *>(sys->d_stage), *dv = dp + 3 * (size_t)n;
  const unsigned g = hb_div_up(n, 256);
  const uint32_t none = 0xFFFFFFFFu;
  if (positions) {
    HB_CUDA(cudaMemcpyAsync(dp, positions, sizeof(T) * 3 * n, cudaMemcpyHostToDevice, s));
    HB_CUDA(cudaMemcpyAsync(sys->d_bad, &none, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    k_state_check<T><<<g, 256, 0, s>>>(dp, sys->d_bad, n);
  }
  if (velocities)
    HB_CUDA(cudaMemcpyAsync(dv, velocities, sizeof(T) * 3 * n, cudaMemcpyHostToDevice, s));
  k_state_in<T><<<g, 256, 0, s>>>(positions ? dp : nullptr, velocities ? dv : nullptr,
                                  sys->d_box64, sys->d_posq, sys->d_vel, sys->d_image,
                                  positions ? sys->d_bad : nullptr, n);
  HB_CUDA(cudaGetLastError());
  uint32_t bad = none;
  if (positions)
    HB_CUDA(cudaMemcpyAsync(&bad, sys->d_bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  // the host arrays may be reused as soon as the call returns
  HB_CUDA(cudaStreamSynchronize(s));
  if (bad != none)
    return hb_fail(HB_ERR_NOT_FINITE, "non-finite position for atom " + std::to_string(bad));
  sys->fix_valid = false;
  return HB_OK;
}

template <class T>
int get_state_t(hb_system *sys, T *positions, T *velocities, int32_t *images, T *forces) {
  HB_REQUIRE(sys, HB_ERR_INVALID_ARGUMENT, "null system");
  const uint32_t n = sys->n;
  if (!n || (!positions && !velocities && !images && !forces)) return HB_OK;
  HB_TRY(stage_alloc(sys));
  cudaStream_t s = sys->ctx->stream;
  // work on the second stream is joined into the first one by every force
  // evaluation; wait for it anyway in case a caller queued some there
  HB_CUDA(cudaStreamSynchronize(sys->ctx->stream2));
  const size_t n3 = 3 * (size_t)n;
  T *dp = reinterpret_cast<T *>(sys->d_stage), *dv = dp + n3, *df = dv + n3;
  k_state_out<T><<<hb_div_up(n, 256), 256, 0, s>>>(
      sys->d_posq, sys->d_vel, sys->d_force, sys->d_image, positions ? dp : nullptr,
      velocities ? dv : nullptr, forces ? df : nullptr, images ? sys->d_stage_img : nullptr, n);
  HB_CUDA(cudaGetLastError());
  if (positions)
    HB_CUDA(cudaMemcpyAsync(positions, dp, sizeof(T) * n3, cudaMemcpyDeviceToHost, s));
  if (velocities)
    HB_CUDA(cudaMemcpyAsync(velocities, dv, sizeof(T) * n3, cudaMemcpyDeviceToHost, s));
  if (forces)
    HB_CUDA(cudaMemcpyAsync(forces, df, sizeof(T) * n3, cudaMemcpyDeviceToHost, s));
  if (images)
    HB_CUDA(cudaMemcpyAsync(images, sys->d_stage_img, sizeof(int32_t) * n3,
                            cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  return HB_OK;
}

}  // namespace

extern "C" int hb_system_set_state(hb_system *sys, const double *positions,
                                   const double *velocities) {
  return set_state_t<double>(sys, positions, velocities);
}

extern "C" int hb_system_get_state(hb_system *sys, double *positions, double *velocities,
                                   int32_t *images, double *forces) {
  return get_state_t<double>(sys, positions, velocities, images, forces);
}

extern "C" int hb_system_set_state_f32(hb_system *sys, const float *positions,
                                       const float *velocities) {
  return set_state_t<float>(sys, positions, velocities);
}

extern "C" int hb_system_get_state_f32(hb_system *sys, float *positions, float *velocities,
                                       int32_t *images, float *forces) {
  return get_state_t<float>(sys, positions, velocities, images, forces);
}

extern "C" int hb_system_set_box(hb_system *sys, const double box[6]) {
  HB_REQUIRE(sys && box, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_REQUIRE(finite6(box), HB_ERR_NOT_FINITE, "box must be finite with positive diagonal");
  std::memcpy(sys->box, box, sizeof(double) * 6);
  DBox db = make_dbox(box);
  HB_CUDA(cudaStreamSynchronize(sys->ctx->stream));
  HB_CUDA(cudaMemcpy(sys->d_box, &db, sizeof(DBox), cudaMemcpyHostToDevice));
  HB_CUDA(cudaMemcpy(sys->d_box64, box, sizeof(double) * 6, cudaMemcpyHostToDevice));
  return HB_OK;
}

extern "C" int hb_system_flip_velocities(hb_system *sys) {
  HB_REQUIRE(sys, HB_ERR_INVALID_ARGUMENT, "null system");
  return integ_flip_velocities(sys, sys->ctx->stream);
}

extern "C" int hb_system_get_box(hb_system *sys, double box[6]) {
  HB_REQUIRE(sys && box, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_TRY(sys_refresh_box(sys));
  std::memcpy(box, sys->box, sizeof(double) * 6);
  return HB_OK;
}

// ---------------------------------------------------------------------
// force field
// ---------------------------------------------------------------------
extern "C" int hb_forcefield_destroy(hb_forcefield *ff) {
  if (!ff) return HB_OK;
  cudaSetDevice(ff->sys->ctx->device);
  hb_context_synchronize(ff->sys->ctx);
  nl_free(ff);
  bonded_free(ff);
  if (ff->spme.on) spme_free(ff);
  cudaFree(ff->d_lj);
  cudaFree(ff->d_lj_invd);
  cudaFree(ff->d_excl_off);
  cudaFree(ff->d_excl_partner);
  cudaFree(ff->d_excl_scale);
  cudaFree(ff->d_scalars);
  cudaFree(ff->d_acc);
  cudaFree(ff->d_energy);
  cudaFree(ff->d_virial);
  delete ff;
  return HB_OK;
}

extern "C" int hb_forcefield_create(hb_system *sys, const hb_forcefield_desc *d,
                                    hb_forcefield **out) {
  HB_REQUIRE(sys && d && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  const uint32_t n = sys->n;
  hb_forcefield tmp;
  double rc_max = 0.0;
  if (d->lj_enabled) {
    HB_REQUIRE(d->n_types >= 1 && d->n_types <= 64, HB_ERR_INVALID_ARGUMENT,
               "LJ needs 1..64 particle types");
    HB_REQUIRE(d->lj_sigma && d->lj_epsilon && d->lj_cutoff && d->lj_switch,
               HB_ERR_INVALID_ARGUMENT, "LJ tables are required");
    for (uint32_t i = 0; i < n; ++i)
      HB_REQUIRE(sys->h_type[i] < d->n_types, HB_ERR_INVALID_ARGUMENT,
                 "particle type index out of range");
    const uint32_t nt2 = d->n_types * d->n_types;
    for (uint32_t k = 0; k < nt2; ++k) {
      const double sg = d->lj_sigma[k], ep = d->lj_epsilon[k], c = d->lj_cutoff[k],
                   sw = d->lj_switch[k];
      HB_REQUIRE(std::isfinite(sg) && std::isfinite(ep) && std::isfinite(c) && std::isfinite(sw),
                 HB_ERR_NOT_FINITE, "LJ parameters must be finite");
      HB_REQUIRE(c > 0.0 && sw > 0.0 && sw <= c, HB_ERR_INVALID_ARGUMENT,
                 "LJ needs 0 < r_switch <= cutoff");
      if (ep != 0.0) rc_max = std::max(rc_max, c);
      if (sw < c) tmp.any_switch = 1;
      tmp.h_lj.push_back(make_float4((float)(sg * sg), (float)(24.0 * ep), (float)(c * c),
                                     (float)(sw * sw)));
    }
    tmp.lj_on = 1;
    tmp.n_types = d->n_types;
  }
  if (d->coulomb_enabled) {
    HB_REQUIRE(std::isfinite(d->alpha) && d->alpha > 0.0 && std::isfinite(d->r_cut_coulomb) &&
                   d->r_cut_coulomb > 0.0,
               HB_ERR_INVALID_ARGUMENT, "Coulomb needs alpha > 0 and r_cut > 0");
    tmp.coul_on = 1;
    tmp.alpha = (float)d->alpha;
    tmp.coul_rc2 = (float)(d->r_cut_coulomb * d->r_cut_coulomb);
    rc_max = std::max(rc_max, d->r_cut_coulomb);
  }
  if (d->recip_enabled) {
    HB_REQUIRE(d->coulomb_enabled, HB_ERR_UNSUPPORTED,
               "SPME reciprocal needs the erfc real-space slot");
    HB_REQUIRE(d->spline_order >= 4 && d->spline_order <= 8, HB_ERR_INVALID_ARGUMENT,
               "spline order must be 4..8");
  }
  HB_REQUIRE(std::isfinite(d->r_skin) && d->r_skin >= 0.0, HB_ERR_INVALID_ARGUMENT,
             "r_skin must be finite and >= 0");
  if (!tmp.lj_on) tmp.n_types = 1;
  if (tmp.h_lj.empty()) tmp.h_lj.push_back(make_float4(0.f, 0.f, 0.f, 0.f));
  tmp.rc_max = (float)rc_max;
  tmp.r_skin = (float)d->r_skin;
  tmp.r_search = (float)(rc_max + d->r_skin);
  // minimum image is well defined only for r_search <= half the smallest
  // perpendicular width (src/integrator/mc_barostat.rs:290-297)
  double w[3];
  HB_TRY(sys_refresh_box(sys));
  perp_widths(sys->box, w);
  const double wmin = std::min(w[0], std::min(w[1], w[2]));
  if ((tmp.lj_on || tmp.coul_on) && n > 1 && wmin < 2.0 * (rc_max + d->r_skin) * (1.0 + 1e-4))
    return hb_fail(HB_ERR_BOX_TOO_SMALL,
                   "box perpendicular width " + std::to_string(wmin) +
                       " is below 2 * (r_cut + r_skin) = " +
                       std::to_string(2.0 * (rc_max + d->r_skin)));
  // exclusions: symmetric CSR with ids in range
  std::vector<uint32_t> eoff, epart;
  std::vector<float2> escale;
  if (d->excl_offsets) {
    HB_REQUIRE(d->excl_offsets[0] == 0, HB_ERR_INVALID_ARGUMENT, "exclusion offsets must start at 0");
    eoff.assign(d->excl_offsets, d->excl_offsets + n + 1);
    const uint32_t ne = eoff[n];
    HB_REQUIRE(ne == 0 || (d->excl_partners && d->excl_lj_scale && d->excl_coulomb_scale),
               HB_ERR_INVALID_ARGUMENT, "exclusion arrays are required");
    std::set<std::pair<uint32_t, uint32_t>> keys;
    for (uint32_t i = 0; i < n; ++i) {
      HB_REQUIRE(eoff[i] <= eoff[i + 1], HB_ERR_INVALID_ARGUMENT, "exclusion offsets must be monotone");
      for (uint32_t q = eoff[i]; q < eoff[i + 1]; ++q) {
        uint32_t j = d->excl_partners[q];
        HB_REQUIRE(j < n && j != i, HB_ERR_INVALID_ARGUMENT, "bad exclusion partner");
        keys.insert({i, j});
        double sl = d->excl_lj_scale[q], sc = d->excl_coulomb_scale[q];
        HB_REQUIRE(std::isfinite(sl) && std::isfinite(sc), HB_ERR_NOT_FINITE, "exclusion scales must be finite");
        if (sl != 0.0 || sc != 0.0) tmp.excl_scaled = 1;
        escale.push_back(make_float2((float)sl, (float)sc));
      }
    }
    for (auto &k : keys)
      HB_REQUIRE(keys.count({k.second, k.first}), HB_ERR_INVALID_ARGUMENT,
                 "exclusion lists must be symmetric");
    epart.assign(d->excl_partners, d->excl_partners + ne);
  }
  HB_REQUIRE(d->pair_mode == HB_PAIRS_FAST || d->pair_mode == HB_PAIRS_EXACT,
             HB_ERR_INVALID_ARGUMENT, "unknown pair_mode");
  hb_forcefield *ff = new hb_forcefield();
  *ff = tmp;
  ff->sys = sys;
  // pair kernel: the balanced queue form (with or without energies); exact
  // pairs take the compacted form with per-pair fixed point and minimum image
  ff->exact_pairs = d->pair_mode == HB_PAIRS_EXACT;
  HB_CUDA(cudaSetDevice(sys->ctx->device));
  HB_CUDA(cudaMalloc(&ff->d_lj, sizeof(float4) * ff->h_lj.size()));
  HB_CUDA(cudaMemcpy(ff->d_lj, ff->h_lj.data(), sizeof(float4) * ff->h_lj.size(),
                     cudaMemcpyHostToDevice));
  {
    std::vector<float> invd(ff->h_lj.size());
    for (size_t q = 0; q < invd.size(); ++q) {
      const float4 L = ff->h_lj[q];
      invd[q] = L.z > L.w ? 1.0f / (L.z - L.w) : 0.0f;
    }
    HB_CUDA(cudaMalloc(&ff->d_lj_invd, sizeof(float) * invd.size()));
    HB_CUDA(cudaMemcpy(ff->d_lj_invd, invd.data(), sizeof(float) * invd.size(),
                       cudaMemcpyHostToDevice));
  }
  if (!eoff.empty()) {
    HB_CUDA(cudaMalloc(&ff->d_excl_off, sizeof(uint32_t) * eoff.size()));
    HB_CUDA(cudaMemcpy(ff->d_excl_off, eoff.data(), sizeof(uint32_t) * eoff.size(), cudaMemcpyHostToDevice));
    const size_t ne = std::max<size_t>(epart.size(), 1);
    HB_CUDA(cudaMalloc(&ff->d_excl_partner, sizeof(uint32_t) * ne));
    HB_CUDA(cudaMalloc(&ff->d_excl_scale, sizeof(float2) * ne));
    if (!epart.empty()) {
      HB_CUDA(cudaMemcpy(ff->d_excl_partner, epart.data(), sizeof(uint32_t) * epart.size(), cudaMemcpyHostToDevice));
      HB_CUDA(cudaMemcpy(ff->d_excl_scale, escale.data(), sizeof(float2) * escale.size(), cudaMemcpyHostToDevice));
    }
    ff->n_excl = (uint32_t)epart.size();
  }
  HB_CUDA(cudaMalloc(&ff->d_scalars, sizeof(double) * HB_N_SCALARS));
  HB_CUDA(cudaMemset(ff->d_scalars, 0, sizeof(double) * HB_N_SCALARS));
  HB_CUDA(cudaMalloc(&ff->d_acc, sizeof(unsigned long long) * 4));
  HB_CUDA(cudaMemset(ff->d_acc, 0, sizeof(unsigned long long) * 4));
  const size_t nn = std::max<size_t>(n, 1);
  HB_CUDA(cudaMalloc(&ff->d_energy, sizeof(float) * nn));
  HB_CUDA(cudaMalloc(&ff->d_virial, sizeof(float) * nn));
  HB_CUDA(cudaMemset(ff->d_energy, 0, sizeof(float) * nn));
  HB_CUDA(cudaMemset(ff->d_virial, 0, sizeof(float) * nn));
  int rc = nl_setup(ff);
  if (rc == HB_OK) rc = bonded_setup(ff, d);
  if (rc == HB_OK && d->recip_enabled) rc = spme_setup(ff, d);
  if (rc == HB_OK) rc = nl_first_build(ff);
  if (rc != HB_OK) {
    std::string msg = g_err;
    hb_forcefield_destroy(ff);
    return hb_fail(rc, msg);
  }
  *out = ff;
  return HB_OK;
}

// ForceField::step body: gated neighbour rebuild, pair kernel on the main
// stream overlapped with the SPME chain on the second stream, combine.
// A force evaluation in three parts: everything before the pair kernel
// (neighbour check / rebuild, tile-order gather, bonded terms, the
// reciprocal-space chain forked onto the second stream), the pair kernel,
// and the join + finalize.  Replica batches put one multi-system pair
// launch between the members' first and last parts.
static int force_pre(hb_forcefield *ff, bool ev, bool capturing) {
  hb_context *ctx = ff->sys->ctx;
  cudaStream_t s = ctx->stream, s2 = ctx->stream2;
  cudaEvent_t t0 = stage_begin(s);
  HB_TRY(nl_displacement_check(ff, s));
  if (capturing) HB_TRY(nl_rebuild_conditional(ff, s));
  else HB_TRY(nl_rebuild(ff, true, s));
  HB_TRY(nl_gather_positions(ff, s));
  stage_end(3, t0, s);
  // bonded terms add into the same fixed-point accumulators (slots of the
  // current list), before the pair kernel on the main stream
  HB_TRY(bonded_launch(ff, ev, s));
  if (ff->spme.on) {
    HB_CUDA(cudaEventRecord(ctx->ev_fork, s));
    HB_CUDA(cudaStreamWaitEvent(s2, ctx->ev_fork, 0));
    cudaEvent_t t2 = stage_begin(s2);
    HB_TRY(spme_launch(ff, ev, s2));
    stage_end(2, t2, s2);
    HB_CUDA(cudaEventRecord(ctx->ev_join, s2));
  }
  return HB_OK;
}

static int force_post(hb_forcefield *ff, bool ev) {
  hb_context *ctx = ff->sys->ctx;
  cudaStream_t s = ctx->stream;
  if (ff->spme.on) HB_CUDA(cudaStreamWaitEvent(s, ctx->ev_join, 0));
  HB_TRY(forces_finalize(ff, ev, s));
  return HB_OK;
}

static int force_eval(hb_forcefield *ff, bool ev, bool capturing = false) {
  cudaStream_t s = ff->sys->ctx->stream;
  HB_TRY(force_pre(ff, ev, capturing));
  cudaEvent_t t1 = stage_begin(s);
  HB_TRY(pair_launch(ff, ev, s));
  stage_end(1, t1, s);
  return force_post(ff, ev);
}

// host check of the status word: overflow is an error (the reference's
// PackedNeighborOverflow), high water grows the buffers
static int check_status(hb_forcefield *ff) {
  cudaStream_t s = ff->sys->ctx->stream;
  HB_CUDA(cudaMemcpyAsync(ff->h_status, ff->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  const uint32_t st = ff->h_status[0];
  if (st & HB_ST_DEVICE_TIMEOUT) {
    // report once; the list is incomplete, so the next step rebuilds it
    const uint32_t clr = (st & ~HB_ST_DEVICE_TIMEOUT) | HB_ST_DISPLACED;
    HB_CUDA(cudaMemcpyAsync(ff->d_status, &clr, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    HB_CUDA(cudaStreamSynchronize(s));
    return hb_fail(HB_ERR_DEVICE_TIMEOUT, "neighbour tile build: a bounded wait for a staged tile gave up");
  }
  if (st & HB_ST_ENTRY_OVERFLOW)
    return hb_fail(HB_ERR_NL_OVERFLOW, "packed neighbour entries overflowed their capacity");
  if (st & HB_ST_ENTRY_HIGHWATER) HB_TRY(nl_first_build(ff));
  return HB_OK;
}

extern "C" int hb_forcefield_step(hb_forcefield *ff, int level) {
  HB_REQUIRE(ff, HB_ERR_INVALID_ARGUMENT, "null force field");
  HB_REQUIRE(level == HB_FORCES_ONLY || level == HB_FORCES_AND_SCALARS, HB_ERR_INVALID_ARGUMENT,
             "bad aggregate level");
  HB_TRY(force_eval(ff, level == HB_FORCES_AND_SCALARS));
  return check_status(ff);
}

extern "C" int hb_forcefield_pre_step(hb_forcefield *ff, int force, int *rebuilt) {
  HB_REQUIRE(ff, HB_ERR_INVALID_ARGUMENT, "null force field");
  cudaStream_t s = ff->sys->ctx->stream;
  uint32_t before = 0, after = 0;
  HB_CUDA(cudaMemcpyAsync(&before, ff->d_counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  if (force) {
    HB_TRY(nl_rebuild(ff, false, s));
  } else {
    HB_TRY(nl_displacement_check(ff, s));
    HB_TRY(nl_rebuild(ff, true, s));
  }
  HB_CUDA(cudaMemcpyAsync(&after, ff->d_counters, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  if (rebuilt) *rebuilt = after != before ? 1 : 0;
  return check_status(ff);
}

extern "C" int hb_forcefield_set_launch(hb_forcefield *ff, int param, int value) {
  HB_REQUIRE(ff, HB_ERR_INVALID_ARGUMENT, "null force field");
  if (param == HB_LAUNCH_PAIR_BLOCKS_PER_SM) {
    HB_REQUIRE(value >= 1 && value <= 8, HB_ERR_INVALID_ARGUMENT, "pair blocks per SM in 1..8");
    ff->pair_blocks_per_sm = value;
  } else if (param == HB_LAUNCH_NL_SLAB) {
    HB_REQUIRE(value >= 2, HB_ERR_INVALID_ARGUMENT, "neighbour slab must hold at least 2 entries");
    HB_TRY(nl_set_slab(ff, (uint32_t)value));
    return check_status(ff);
  } else if (param == HB_LAUNCH_NL_WAIT_TEST) {
    HB_REQUIRE(value >= 0, HB_ERR_INVALID_ARGUMENT, "poll limit must be >= 0");
    ff->nl_polls = value > 0 ? (uint32_t)value : (1u << 20);
    ff->nl_issue = value > 0 ? 0u : 1u;
  } else if (param == HB_LAUNCH_PAIR_QUOTA) {
    HB_REQUIRE(value >= 0 && value <= 4096, HB_ERR_INVALID_ARGUMENT, "pair work quota in 0..4096");
    ff->pair_quota = value;
  } else if (param == HB_LAUNCH_PAIR_CHUNK) {
    HB_REQUIRE(value >= 1 && value <= 64, HB_ERR_INVALID_ARGUMENT, "pair entry chunk in 1..64");
    ff->pair_chunk = value;
  } else if (param == HB_LAUNCH_FFT_PLANE || param == HB_LAUNCH_GATHER_FORM) {
    HB_TRY(spme_set_form(ff, param, value));
  } else {
    return hb_fail(HB_ERR_INVALID_ARGUMENT, "unknown launch parameter");
  }
  ff->layout_gen++;  // launch shapes are baked into captured graphs
  return HB_OK;
}

extern "C" int hb_forcefield_scalars(hb_forcefield *ff, double out[HB_N_SCALARS]) {
  HB_REQUIRE(ff && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_CUDA(cudaStreamSynchronize(ff->sys->ctx->stream));
  HB_CUDA(cudaMemcpy(out, ff->d_scalars, sizeof(double) * HB_N_SCALARS, cudaMemcpyDeviceToHost));
  return HB_OK;
}

extern "C" int hb_forcefield_get_per_atom(hb_forcefield *ff, double *energy, double *virial) {
  HB_REQUIRE(ff, HB_ERR_INVALID_ARGUMENT, "null force field");
  HB_CUDA(cudaStreamSynchronize(ff->sys->ctx->stream));
  const uint32_t n = ff->sys->n;
  std::vector<float> b(std::max(n, 1u));
  if (energy && n) {
    HB_CUDA(cudaMemcpy(b.data(), ff->d_energy, sizeof(float) * n, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < n; ++i) energy[i] = b[i];
  }
  if (virial && n) {
    HB_CUDA(cudaMemcpy(b.data(), ff->d_virial, sizeof(float) * n, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < n; ++i) virial[i] = b[i];
  }
  return HB_OK;
}

extern "C" int hb_neighbor_pairs(hb_forcefield *ff, uint32_t *pairs, uint64_t cap,
                                 uint64_t *count, uint64_t *duplicates) {
  HB_REQUIRE(ff && count, HB_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<uint32_t> p;
  uint64_t dups = 0;
  HB_TRY(nl_pairs(ff, p, dups));
  const uint64_t cnt = p.size() / 2;
  *count = cnt;
  if (duplicates) *duplicates = dups;
  if (pairs) std::memcpy(pairs, p.data(), sizeof(uint32_t) * 2 * std::min(cnt, cap));
  return HB_OK;
}

extern "C" int hb_neighbor_stats(hb_forcefield *ff, uint64_t out[6]) {
  HB_REQUIRE(ff && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  cudaStream_t s = ff->sys->ctx->stream;
  uint32_t cnt[4] = {0, 0, 0, 0}, st = 0;
  HB_CUDA(cudaMemcpyAsync(cnt, ff->d_counters, sizeof(uint32_t) * 4, cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaMemcpyAsync(&st, ff->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  const uint32_t total = cnt[1];
  out[0] = ff->n_tiles;
  out[1] = total;
  out[2] = ff->entry_cap;
  out[3] = cnt[0];
  out[4] = st;
  out[5] = (uint64_t)total * 32u * 32u;
  return HB_OK;
}

extern "C" int hb_neighbor_capacity(hb_forcefield *ff, uint64_t out[4]) {
  HB_REQUIRE(ff && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  cudaStream_t s = ff->sys->ctx->stream;
  std::vector<uint32_t> nent(ff->n_tiles);
  uint32_t st = 0;
  if (ff->n_tiles)
    HB_CUDA(cudaMemcpyAsync(nent.data(), ff->d_tile_nent, sizeof(uint32_t) * ff->n_tiles,
                            cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaMemcpyAsync(&st, ff->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  uint32_t mx = 0;
  for (uint32_t v : nent) mx = std::max(mx, v);
  out[0] = ff->slab;
  out[1] = mx;
  out[2] = ff->reallocations;
  out[3] = st;
  return HB_OK;
}

// ---------------------------------------------------------------------
// constraints
// ---------------------------------------------------------------------
extern "C" int hb_constraints_destroy(hb_constraints *c) {
  if (!c) return HB_OK;
  cudaSetDevice(c->sys->ctx->device);
  cudaStreamSynchronize(c->sys->ctx->stream);
  cudaFree(c->d_settle_atoms);
  cudaFree(c->d_settle_geom);
  cudaFree(c->d_settle_mass);
  cudaFree(c->d_shake_aoff);
  cudaFree(c->d_shake_atoms);
  cudaFree(c->d_shake_coff);
  cudaFree(c->d_shake_pairs);
  cudaFree(c->d_shake_d2);
  cudaFree(c->d_virial);
  cudaFree(c->d_iters);
  cudaFree(c->d_feat);
  cudaFree(c->d_lam1);
  cudaFree(c->d_lsc);
  cudaFree(c->d_lam);
  cudaFree(c->d_pred);
  cudaFree(c->d_stats);
  delete c;
  return HB_OK;
}

extern "C" int hb_constraints_create(hb_system *sys, const hb_constraints_desc *d,
                                     hb_constraints **out) {
  HB_REQUIRE(sys && d && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  const uint32_t n = sys->n, ng = d->n_groups;
  HB_REQUIRE(ng == 0 || (d->group_offsets && d->group_atoms && d->group_kind),
             HB_ERR_INVALID_ARGUMENT, "group arrays are required");
  std::vector<uint4> s_atoms;
  std::vector<float4> s_geom;
  std::vector<float2> s_mass;
  std::vector<uint32_t> h_aoff{0}, h_atoms, h_coff{0};
  std::vector<uint2> h_pairs;
  std::vector<double> h_d2;
  std::vector<char> seen(n, 0);
  for (uint32_t g = 0; g < ng; ++g) {
    const uint32_t a0 = d->group_offsets[g], a1 = d->group_offsets[g + 1];
    HB_REQUIRE(a1 > a0, HB_ERR_CONSTRAINT_SHAPE, "empty constraint group");
    for (uint32_t a = a0; a < a1; ++a) {
      const uint32_t id = d->group_atoms[a];
      HB_REQUIRE(id < n, HB_ERR_CONSTRAINT_SHAPE, "constraint atom out of range");
      HB_REQUIRE(!seen[id], HB_ERR_CONSTRAINT_SHAPE, "an atom belongs to two constraint groups");
      seen[id] = 1;
    }
    if (d->group_kind[g] == HB_CONSTRAINT_SETTLE) {
      HB_REQUIRE(a1 - a0 == 3, HB_ERR_CONSTRAINT_SHAPE, "SETTLE groups hold exactly 3 atoms (O, H, H)");
      HB_REQUIRE(d->settle_ra && d->settle_rb && d->settle_rc, HB_ERR_INVALID_ARGUMENT,
                 "SETTLE geometry is required");
      const uint32_t o = d->group_atoms[a0], h1 = d->group_atoms[a0 + 1], h2 = d->group_atoms[a0 + 2];
      HB_REQUIRE(sys->h_mass[h1] == sys->h_mass[h2], HB_ERR_CONSTRAINT_SHAPE,
                 "SETTLE needs equal hydrogen masses");
      s_atoms.push_back(make_uint4(o, h1, h2, 0));
      s_geom.push_back(make_float4((float)d->settle_ra[g], (float)d->settle_rb[g],
                                   (float)d->settle_rc[g], 0.f));
      s_mass.push_back(make_float2((float)sys->h_mass[o], (float)sys->h_mass[h1]));
    } else if (d->group_kind[g] == HB_CONSTRAINT_SHAKE) {
      HB_REQUIRE(a1 - a0 <= 8, HB_ERR_CONSTRAINT_SHAPE, "SHAKE groups hold at most 8 atoms");
      HB_REQUIRE(d->con_offsets && d->con_i && d->con_j && d->con_dist, HB_ERR_INVALID_ARGUMENT,
                 "SHAKE constraints are required");
      const uint32_t c0 = d->con_offsets[g], c1 = d->con_offsets[g + 1];
      HB_REQUIRE(c1 >= c0 && c1 - c0 <= 12, HB_ERR_CONSTRAINT_SHAPE,
                 "SHAKE groups hold at most 12 constraints");
      for (uint32_t a = a0; a < a1; ++a) h_atoms.push_back(d->group_atoms[a]);
      h_aoff.push_back((uint32_t)h_atoms.size());
      for (uint32_t k = c0; k < c1; ++k) {
        HB_REQUIRE(d->con_i[k] < a1 - a0 && d->con_j[k] < a1 - a0 && d->con_i[k] != d->con_j[k],
                   HB_ERR_CONSTRAINT_SHAPE, "bad SHAKE constraint pair");
        HB_REQUIRE(std::isfinite(d->con_dist[k]) && d->con_dist[k] > 0.0, HB_ERR_CONSTRAINT_SHAPE,
                   "SHAKE distances must be positive");
        h_pairs.push_back(make_uint2(d->con_i[k], d->con_j[k]));
        h_d2.push_back(d->con_dist[k] * d->con_dist[k]);
      }
      h_coff.push_back((uint32_t)h_pairs.size());
    } else {
      return hb_fail(HB_ERR_CONSTRAINT_SHAPE, "unknown constraint kind");
    }
  }
  hb_constraints *c = new hb_constraints();
  c->sys = sys;
  c->n_settle = (uint32_t)s_atoms.size();
  c->n_shake = (uint32_t)h_aoff.size() - 1;
  if (d->shake_tol > 0.0) c->shake_tol = d->shake_tol;
  if (d->shake_max_iter > 0) c->shake_max_iter = d->shake_max_iter;
  c->shake_rel = d->shake_tol_relative ? 1 : 0;
  c->n_shake_cons = (uint32_t)h_pairs.size();
  auto up = [](void **dst, const void *src, size_t bytes) -> int {
    HB_CUDA(cudaMalloc(dst, std::max<size_t>(bytes, 16)));
    if (bytes) HB_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    return HB_OK;
  };
  int rc = HB_OK;
  if (rc == HB_OK) rc = up((void **)&c->d_settle_atoms, s_atoms.data(), sizeof(uint4) * s_atoms.size());
  if (rc == HB_OK) rc = up((void **)&c->d_settle_geom, s_geom.data(), sizeof(float4) * s_geom.size());
  if (rc == HB_OK) rc = up((void **)&c->d_settle_mass, s_mass.data(), sizeof(float2) * s_mass.size());
  if (rc == HB_OK) rc = up((void **)&c->d_shake_aoff, h_aoff.data(), sizeof(uint32_t) * h_aoff.size());
  if (rc == HB_OK) rc = up((void **)&c->d_shake_atoms, h_atoms.data(), sizeof(uint32_t) * h_atoms.size());
  if (rc == HB_OK) rc = up((void **)&c->d_shake_coff, h_coff.data(), sizeof(uint32_t) * h_coff.size());
  if (rc == HB_OK) rc = up((void **)&c->d_shake_pairs, h_pairs.data(), sizeof(uint2) * h_pairs.size());
  if (rc == HB_OK) rc = up((void **)&c->d_shake_d2, h_d2.data(), sizeof(double) * h_d2.size());
  if (rc == HB_OK) {
    const size_t nn = std::max<size_t>(n, 1);
    if (cudaMalloc(&c->d_virial, sizeof(float) * nn) != cudaSuccess ||
        cudaMemset(c->d_virial, 0, sizeof(float) * nn) != cudaSuccess ||
        cudaMalloc(&c->d_iters, sizeof(uint32_t)) != cudaSuccess ||
        cudaMemset(c->d_iters, 0, sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&c->d_stats, sizeof(unsigned long long) * 2) != cudaSuccess ||
        cudaMemset(c->d_stats, 0, sizeof(unsigned long long) * 2) != cudaSuccess)
      rc = hb_fail(HB_ERR_CUDA, "constraint buffer allocation failed");
    const size_t m = std::max<size_t>(c->n_shake_cons, 1);
    if (rc == HB_OK &&
        (cudaMalloc(&c->d_feat, sizeof(float) * 8 * m) != cudaSuccess ||
         cudaMalloc(&c->d_lam1, sizeof(double) * m) != cudaSuccess ||
         cudaMalloc(&c->d_lsc, sizeof(double) * m) != cudaSuccess ||
         cudaMalloc(&c->d_lam, sizeof(double) * m) != cudaSuccess ||
         cudaMalloc(&c->d_pred, sizeof(float) * m) != cudaSuccess ||
         cudaMemset(c->d_feat, 0, sizeof(float) * 8 * m) != cudaSuccess ||
         cudaMemset(c->d_lam1, 0, sizeof(double) * m) != cudaSuccess ||
         cudaMemset(c->d_lsc, 0, sizeof(double) * m) != cudaSuccess ||
         cudaMemset(c->d_lam, 0, sizeof(double) * m) != cudaSuccess))
      rc = hb_fail(HB_ERR_CUDA, "constraint buffer allocation failed");
  }
  if (rc != HB_OK) {
    hb_constraints_destroy(c);
    return rc;
  }
  *out = c;
  return HB_OK;
}

extern "C" int hb_constraints_shake_stats(hb_constraints *c, double out[3], int reset) {
  HB_REQUIRE(c && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  unsigned long long s[2] = {0, 0};
  HB_CUDA(cudaStreamSynchronize(c->sys->ctx->stream));
  HB_CUDA(cudaMemcpy(s, c->d_stats, sizeof(s), cudaMemcpyDeviceToHost));
  out[0] = (double)s[0];
  out[1] = (double)s[1];
  out[2] = s[1] ? (double)s[0] / (double)s[1] : 0.0;
  if (reset) HB_CUDA(cudaMemset(c->d_stats, 0, sizeof(s)));
  return HB_OK;
}

extern "C" int hb_constraints_record(hb_constraints *c, int enable) {
  HB_REQUIRE(c, HB_ERR_INVALID_ARGUMENT, "null constraints");
  c->record = enable != 0;
  return HB_OK;
}

extern "C" int hb_constraints_fuse_head(hb_constraints *c, int enable) {
  HB_REQUIRE(c, HB_ERR_INVALID_ARGUMENT, "null constraints");
  if (c->fuse_head != (enable != 0)) {
    c->fuse_head = enable != 0;
    c->uid = hb_next_uid();  // graphs captured with the other form are stale
  }
  return HB_OK;
}

extern "C" int hb_constraints_get_record(hb_constraints *c, float *features, double *lam1,
                                         double *lscale, double *lam, uint32_t *m) {
  HB_REQUIRE(c, HB_ERR_INVALID_ARGUMENT, "null constraints");
  if (m) *m = c->n_shake_cons;
  const size_t k = c->n_shake_cons;
  if (!k) return HB_OK;
  HB_CUDA(cudaStreamSynchronize(c->sys->ctx->stream));
  if (features) HB_CUDA(cudaMemcpy(features, c->d_feat, sizeof(float) * 8 * k, cudaMemcpyDeviceToHost));
  if (lam1) HB_CUDA(cudaMemcpy(lam1, c->d_lam1, sizeof(double) * k, cudaMemcpyDeviceToHost));
  if (lscale) HB_CUDA(cudaMemcpy(lscale, c->d_lsc, sizeof(double) * k, cudaMemcpyDeviceToHost));
  if (lam) HB_CUDA(cudaMemcpy(lam, c->d_lam, sizeof(double) * k, cudaMemcpyDeviceToHost));
  return HB_OK;
}

extern "C" int hb_constraints_set_warm_start(hb_constraints *c, hb_shake_mlp *m) {
  HB_REQUIRE(c, HB_ERR_INVALID_ARGUMENT, "null constraints");
  c->mlp = m;
  return HB_OK;
}

extern "C" int hb_constraints_before_drift(hb_constraints *c) {
  HB_REQUIRE(c, HB_ERR_INVALID_ARGUMENT, "null constraints");
  c->sys->fix_valid = false;
  hb_system *sys = c->sys;
  if (sys->n)
    HB_CUDA(cudaMemcpyAsync(sys->d_pos_prev, sys->d_posq, sizeof(float4) * sys->n,
                            cudaMemcpyDeviceToDevice, sys->ctx->stream));
  return HB_OK;
}

extern "C" int hb_constraints_after_drift(hb_constraints *c, double dt) {
  HB_REQUIRE(c, HB_ERR_INVALID_ARGUMENT, "null constraints");
  c->sys->fix_valid = false;
  return cons_positions(c, dt, c->sys->ctx->stream);
}

extern "C" int hb_constraints_after_kick(hb_constraints *c, double dt) {
  HB_REQUIRE(c, HB_ERR_INVALID_ARGUMENT, "null constraints");
  c->sys->fix_valid = false;
  return cons_velocities(c, dt, dt > 0.0, c->sys->ctx->stream);
}

extern "C" int hb_constraints_get_virial(hb_constraints *c, double *virial) {
  HB_REQUIRE(c && virial, HB_ERR_INVALID_ARGUMENT, "null argument");
  const uint32_t n = c->sys->n;
  HB_CUDA(cudaStreamSynchronize(c->sys->ctx->stream));
  std::vector<float> b(std::max(n, 1u));
  if (n) HB_CUDA(cudaMemcpy(b.data(), c->d_virial, sizeof(float) * n, cudaMemcpyDeviceToHost));
  for (uint32_t i = 0; i < n; ++i) virial[i] = b[i];
  return HB_OK;
}

// ---------------------------------------------------------------------
// integrator
// ---------------------------------------------------------------------
extern "C" int hb_integrator_create(hb_system *sys, const hb_integrator_desc *d,
                                    hb_integrator **out) {
  HB_REQUIRE(sys && d && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_REQUIRE(d->kind == HB_INTEGRATOR_VV || d->kind == HB_INTEGRATOR_VV_LOSSLESS ||
                 d->kind == HB_INTEGRATOR_LANGEVIN,
             HB_ERR_INVALID_ARGUMENT, "unknown integrator kind");
  HB_REQUIRE(std::isfinite(d->dt) && d->dt > 0.0, HB_ERR_INVALID_ARGUMENT, "dt must be > 0");
  if (d->kind == HB_INTEGRATOR_LANGEVIN)
    HB_REQUIRE(std::isfinite(d->friction) && d->friction > 0.0 && std::isfinite(d->temperature) &&
                   d->temperature > 0.0,
               HB_ERR_INVALID_ARGUMENT, "Langevin needs friction > 0 and temperature > 0");
  hb_integrator *it = new hb_integrator();
  it->sys = sys;
  it->kind = d->kind;
  it->dt = d->dt;
  it->friction = d->friction;
  it->temperature = d->temperature;
  it->seed = d->seed;
  it->step = d->step0;
  if (cudaMalloc(&it->d_step, sizeof(uint64_t)) != cudaSuccess ||
      cudaMemcpy(it->d_step, &it->step, sizeof(uint64_t), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMalloc(&it->d_done, sizeof(uint32_t)) != cudaSuccess ||
      cudaMemset(it->d_done, 0, sizeof(uint32_t)) != cudaSuccess ||
      cudaEventCreate(&it->g_ev0) != cudaSuccess || cudaEventCreate(&it->g_ev1) != cudaSuccess) {
    hb_integrator_destroy(it);
    return hb_fail(HB_ERR_CUDA, "integrator state allocation failed");
  }
  if (it->kind == HB_INTEGRATOR_VV_LOSSLESS) {
    // the fixed-point state starts from the current f32 state (snapped to it)
    int rc = integ_fix_derive(sys, sys->ctx->stream);
    if (rc == HB_OK && cudaStreamSynchronize(sys->ctx->stream) != cudaSuccess) rc = HB_ERR_CUDA;
    if (rc != HB_OK) {
      hb_integrator_destroy(it);
      return hb_fail(rc, "lossless state initialisation failed");
    }
  }
  *out = it;
  return HB_OK;
}

extern "C" int hb_integrator_destroy(hb_integrator *it) {
  if (!it) return HB_OK;
  cudaStreamSynchronize(it->sys->ctx->stream);
  if (it->graph_exec) cudaGraphExecDestroy(it->graph_exec);
  if (it->graph_exec_move) cudaGraphExecDestroy(it->graph_exec_move);
  if (it->graph_exec_x) cudaGraphExecDestroy(it->graph_exec_x);
  if (it->graph_exec_x_move) cudaGraphExecDestroy(it->graph_exec_x_move);
  cudaFree(it->d_step);
  cudaFree(it->d_done);
  if (it->g_ev0) cudaEventDestroy(it->g_ev0);
  if (it->g_ev1) cudaEventDestroy(it->g_ev1);
  delete it;
  return HB_OK;
}

// One step.  Velocity Verlet keeps the reference's hook order
// (src/integrator/mod.rs:344-429 with the post-force kick of
// src/runner.rs:2673-2686): snapshot, kick-drift, position constraint,
// forces, velocity projection, final half kick.  Langevin (middle scheme):
// full kick, velocity projection, half drift, O, half drift, position
// constraint, forces.
// One MD step = step_head (kicks, drift, constraint positions), a force
// evaluation with energies when step_force_ev says so, and step_tail (the
// velocity-Verlet final kick with its constraint and coupling parts).
static int step_head(hb_integrator *it, hb_constraints *cons) {
  cudaStream_t s = it->sys->ctx->stream;
  cudaEvent_t t4 = stage_begin(s);
  if (it->kind == HB_INTEGRATOR_LANGEVIN && cons_lang_head_fusable(cons)) {
    // every atom in a SETTLE water: the four parts in one kernel
    HB_TRY(cons_lang_settle_head(cons, (float)it->dt, (float)std::exp(-it->friction * it->dt),
                                 (float)it->temperature, (uint32_t)it->seed,
                                 (uint32_t)(it->seed >> 32), it->d_step, it->d_done, s));
  } else if (it->kind == HB_INTEGRATOR_LANGEVIN) {
    HB_TRY(integ_lang_kick(it, s));
    if (cons) HB_TRY(cons_velocities(cons, 0.0, false, s));
    HB_TRY(integ_lang_drift_ou(it, s));
    if (cons) HB_TRY(cons_positions(cons, it->dt, s));
  } else {
    HB_TRY(integ_vv_kick_drift(it, s));
    if (cons) HB_TRY(cons_positions(cons, it->dt, s));
  }
  stage_end(4, t4, s);
  return HB_OK;
}

// per-step pressure coupling reads the virial of every step
static bool step_force_ev(const hb_integrator *it, bool ev) {
  return it->kind == HB_INTEGRATOR_LANGEVIN ? ev : (ev || it->pc != nullptr);
}

static int step_tail(hb_integrator *it, hb_forcefield *ff, hb_constraints *cons) {
  cudaStream_t s = it->sys->ctx->stream;
  if (it->kind != HB_INTEGRATOR_LANGEVIN) {
    cudaEvent_t t5 = stage_begin(s);
    if (cons) HB_TRY(cons_velocities(cons, it->dt, true, s));
    if (it->thermo || it->pc) {
      HB_TRY(couple_prepare(it, ff, cons, s));
      HB_TRY(couple_final_kick(it, s));
    } else {
      HB_TRY(integ_vv_kick(it, s));
    }
    stage_end(4, t5, s);
  }
  it->step++;
  return HB_OK;
}

static int one_step(hb_integrator *it, hb_forcefield *ff, hb_constraints *cons, bool ev,
                    bool capturing = false) {
  HB_TRY(step_head(it, cons));
  HB_TRY(force_eval(ff, step_force_ev(it, ev), capturing));
  return step_tail(it, ff, cons);
}

// Barostat::apply_move on the device: propose + scale, a forces + scalars
// evaluation against the trial box, Metropolis test + revert.
static int baro_move(hb_barostat *b, hb_forcefield *ff, bool capturing) {
  cudaStream_t s = ff->sys->ctx->stream;
  HB_TRY(baro_propose(b, ff, s));
  HB_TRY(force_eval(ff, true, capturing));
  HB_TRY(baro_decide(b, ff, s));
  return HB_OK;
}

extern "C" int hb_barostat_mc_move(hb_barostat *b, hb_forcefield *ff) {
  HB_REQUIRE(b && ff, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_REQUIRE(ff->sys == b->sys, HB_ERR_INVALID_ARGUMENT,
             "barostat and force field must share one system");
  if (b->sys->n == 0) return HB_OK;
  b->sys->fix_valid = false;
  HB_TRY(baro_move(b, ff, false));
  return check_status(ff);
}

// ---------------------------------------------------------------------
// steepest-descent minimiser
// ---------------------------------------------------------------------
extern "C" int hb_minimizer_create(hb_forcefield *ff, hb_constraints *cons,
                                   const hb_minimizer_desc *d, hb_minimizer **out) {
  HB_REQUIRE(ff && d && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_REQUIRE(!cons || cons->sys == ff->sys, HB_ERR_INVALID_ARGUMENT,
             "force field and constraints must share one system");
  // the reference's schema checks (steepest_descent.rs:300-380)
  HB_REQUIRE(std::isfinite(d->initial_step) && d->initial_step > 0.0, HB_ERR_INVALID_ARGUMENT,
             "minimization.algorithm.initial_step: expected finite and strictly positive");
  HB_REQUIRE(std::isfinite(d->max_step) && d->max_step > 0.0, HB_ERR_INVALID_ARGUMENT,
             "minimization.algorithm.max_step: expected finite and strictly positive");
  HB_REQUIRE(d->max_step >= d->initial_step, HB_ERR_INVALID_ARGUMENT,
             "minimization.algorithm.max_step must be >= initial_step");
  HB_REQUIRE(std::isfinite(d->step_increase) && d->step_increase >= 1.0, HB_ERR_INVALID_ARGUMENT,
             "minimization.algorithm.step_increase must be finite and >= 1.0");
  HB_REQUIRE(std::isfinite(d->step_decrease) && d->step_decrease > 0.0 && d->step_decrease < 1.0,
             HB_ERR_INVALID_ARGUMENT,
             "minimization.algorithm.step_decrease must be finite and in (0.0, 1.0)");
  HB_REQUIRE(std::isfinite(d->force_tolerance) && d->force_tolerance >= 0.0,
             HB_ERR_INVALID_ARGUMENT,
             "minimization.algorithm.force_tolerance must be finite and >= 0.0");
  HB_REQUIRE(std::isfinite(d->energy_tolerance) && d->energy_tolerance >= 0.0,
             HB_ERR_INVALID_ARGUMENT,
             "minimization.algorithm.energy_tolerance must be finite and >= 0.0");
  HB_REQUIRE(d->max_iterations > 0, HB_ERR_INVALID_ARGUMENT,
             "minimization.algorithm.max_iterations must be strictly positive");
  hb_minimizer *m = new hb_minimizer();
  m->ff = ff;
  m->cons = cons;
  m->initial_step = (float)d->initial_step;
  m->max_step = (float)d->max_step;
  m->inc = (float)d->step_increase;
  m->dec = (float)d->step_decrease;
  m->ftol = d->force_tolerance;
  m->etol = d->energy_tolerance;
  m->max_iter = d->max_iterations;
  const int rc = min_alloc(m);
  if (rc != HB_OK) {
    std::string msg = hb_last_error();
    hb_minimizer_destroy(m);
    return hb_fail(rc, msg);
  }
  *out = m;
  return HB_OK;
}

extern "C" int hb_minimizer_destroy(hb_minimizer *m) {
  if (!m) return HB_OK;
  cudaStreamSynchronize(m->ff->sys->ctx->stream);
  min_free(m);
  delete m;
  return HB_OK;
}

extern "C" int hb_minimizer_begin(hb_minimizer *m, hb_min_report *out) {
  HB_REQUIRE(m && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  hb_forcefield *ff = m->ff;
  cudaStream_t s = ff->sys->ctx->stream;
  ff->sys->fix_valid = false;
  HB_TRY(force_eval(ff, true));
  HB_TRY(min_init(m, s));
  HB_CUDA(cudaMemcpyAsync(out, m->d_rep, sizeof(hb_min_report), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  HB_TRY(check_status(ff));
  m->begun = true;
  m->done = 0;
  m->converged = out->converged;
  return HB_OK;
}

extern "C" int hb_minimizer_iterate(hb_minimizer *m, uint32_t n, hb_min_report *out,
                                    uint32_t *n_done) {
  HB_REQUIRE(m && n_done && (out || n == 0), HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_REQUIRE(m->begun, HB_ERR_INVALID_ARGUMENT, "hb_minimizer_begin must come first");
  *n_done = 0;
  hb_forcefield *ff = m->ff;
  cudaStream_t s = ff->sys->ctx->stream;
  ff->sys->fix_valid = false;
  while (n > 0 && !m->converged && m->done < m->max_iter) {
    uint32_t chunk = std::min<uint64_t>({(uint64_t)n, (uint64_t)m->rep_cap, m->max_iter - m->done});
    MinState before, after;
    HB_CUDA(cudaMemcpyAsync(&before, m->d_st, sizeof(MinState), cudaMemcpyDeviceToHost, s));
    for (uint32_t k = 0; k < chunk; ++k) {
      HB_TRY(min_trial(m, s));
      if (m->cons) HB_TRY(cons_project(m->cons, &m->d_st->skip, s));
      HB_TRY(force_eval(ff, true));
      HB_TRY(min_finish(m, k, s));
    }
    HB_CUDA(cudaMemcpyAsync(&after, m->d_st, sizeof(MinState), cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    const uint32_t got = (uint32_t)(after.iteration - before.iteration);
    if (got)
      HB_CUDA(cudaMemcpy(out + *n_done, m->d_rep, sizeof(hb_min_report) * got,
                         cudaMemcpyDeviceToHost));
    HB_TRY(check_status(ff));
    *n_done += got;
    m->done += got;
    n -= chunk;
    m->converged = after.converged;
    if (got < chunk && !after.converged) break;  // F_max = 0 at a rejected state
  }
  return HB_OK;
}

extern "C" int hb_integrator_set_barostat(hb_integrator *it, hb_barostat *b) {
  HB_REQUIRE(it, HB_ERR_INVALID_ARGUMENT, "null integrator");
  HB_REQUIRE(!b || b->sys == it->sys, HB_ERR_INVALID_ARGUMENT,
             "integrator and barostat must share one system");
  HB_REQUIRE(!b || !it->pc, HB_ERR_UNSUPPORTED,
             "one barostat per integrator: detach the pressure coupling first");
  it->baro = b;
  return HB_OK;
}

// a move follows the step whose number (counted from 1) is a multiple of
// the barostat's frequency (src/runner.rs:2606-2607, 2693-2708)
static bool move_due(const hb_integrator *it, uint64_t step_number) {
  return it->baro && it->sys->n && step_number % it->baro->frequency == 0;
}

// Lossless mode keeps its own fixed-point state: it takes no constraints or
// barostat (the reference's lossless integrator rejects constraints,
// src/integrator/mod.rs:652) and re-derives the state when something else
// wrote positions or velocities; any other integrator invalidates it.
static int lossless_prologue(hb_integrator *it, hb_constraints *cons) {
  hb_system *sys = it->sys;
  if (it->kind != HB_INTEGRATOR_VV_LOSSLESS) {
    sys->fix_valid = false;
    return HB_OK;
  }
  HB_REQUIRE(!cons, HB_ERR_UNSUPPORTED, "the lossless integrator does not support constraints");
  HB_REQUIRE(!it->baro, HB_ERR_UNSUPPORTED, "the lossless integrator does not support a barostat");
  if (!sys->fix_valid) HB_TRY(integ_fix_derive(sys, sys->ctx->stream));
  return HB_OK;
}

extern "C" int hb_integrator_step(hb_integrator *it, hb_forcefield *ff, hb_constraints *cons,
                                  uint32_t n_steps, uint32_t scalar_every) {
  HB_REQUIRE(it && ff, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_REQUIRE(ff->sys == it->sys && (!cons || cons->sys == it->sys), HB_ERR_INVALID_ARGUMENT,
             "integrator, force field and constraints must share one system");
  HB_TRY(lossless_prologue(it, cons));
  hb_context *ctx = it->sys->ctx;
  StageTimer timer{ctx, {}, 0};
  if (ctx->timing) g_timer = &timer;
  cudaEvent_t t_all = stage_begin(ctx->stream);
  int rc = HB_OK;
  if (!it->forces_valid) {
    rc = force_eval(ff, false);
    it->forces_valid = rc == HB_OK;
  }
  for (uint32_t k = 0; k < n_steps && rc == HB_OK; ++k) {
    const bool move = move_due(it, it->step + 1);
    const bool ev = (scalar_every > 0 && ((k + 1) % scalar_every == 0)) || move;
    rc = one_step(it, ff, cons, ev);
    if (rc == HB_OK && move) rc = baro_move(it->baro, ff, false);
  }
  stage_end(0, t_all, ctx->stream);
  g_timer = nullptr;
  if (rc != HB_OK) return rc;
  HB_TRY(check_status(ff));
  if (cons && cons->mlp) HB_TRY(mlp_status(cons->mlp));
  if (ctx->timing) {
    HB_CUDA(cudaStreamSynchronize(ctx->stream));
    HB_CUDA(cudaStreamSynchronize(ctx->stream2));
    for (int q = 0; q < 8; ++q) ctx->t_ms[q] = 0.0;
    for (auto &m : timer.marks) {
      float ms = 0.f;
      HB_CUDA(cudaEventElapsedTime(&ms, m.second.first, m.second.second));
      ctx->t_ms[m.first] += ms;
    }
  }
  return HB_OK;
}

// capture one step (and, for the move graph, the volume move after it)
static int capture_step(hb_integrator *it, hb_forcefield *ff, hb_constraints *cons, bool move,
                        cudaGraphExec_t *exec) {
  cudaStream_t s = it->sys->ctx->stream;
  cudaGraph_t g;
  HB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const uint64_t step = it->step;
  int rc = one_step(it, ff, cons, move, true);
  if (rc == HB_OK && move) rc = baro_move(it->baro, ff, true);
  it->step = step;
  cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (rc != HB_OK) return rc;
  if (ce != cudaSuccess) return hb_fail(HB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
  cudaError_t ie = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) return hb_fail(HB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
  return HB_OK;
}

static void drop_exchange_graphs(hb_integrator *it) {
  if (it->graph_exec_x) cudaGraphExecDestroy(it->graph_exec_x);
  if (it->graph_exec_x_move) cudaGraphExecDestroy(it->graph_exec_x_move);
  it->graph_exec_x = nullptr;
  it->graph_exec_x_move = nullptr;
  for (auto &k : it->graph_x_key) k = nullptr;
}

static void drop_graphs(hb_integrator *it) {
  if (it->graph_exec) cudaGraphExecDestroy(it->graph_exec);
  if (it->graph_exec_move) cudaGraphExecDestroy(it->graph_exec_move);
  it->graph_exec = nullptr;
  it->graph_exec_move = nullptr;
  drop_exchange_graphs(it);
}

// the graphs of the plain step (and of the step with a volume move), captured
// again whenever an attached object or the force field's buffers changed
static int ensure_step_graphs(hb_integrator *it, hb_forcefield *ff, hb_constraints *cons) {
  const uint64_t cons_uid = cons ? cons->uid : 0, baro_uid = it->baro ? it->baro->uid : 0;
  const uint64_t thermo_uid = it->thermo ? it->thermo->uid : 0, pc_uid = it->pc ? it->pc->uid : 0;
  if (it->graph_exec && it->graph_ff == ff->uid && it->graph_cons == cons_uid &&
      it->graph_baro == baro_uid && it->graph_gen == ff->layout_gen &&
      it->graph_thermo == thermo_uid && it->graph_pc == pc_uid)
    return HB_OK;
  drop_graphs(it);
  HB_CUDA(cudaStreamSynchronize(it->sys->ctx->stream));
  HB_TRY(capture_step(it, ff, cons, false, &it->graph_exec));
  if (it->baro) HB_TRY(capture_step(it, ff, cons, true, &it->graph_exec_move));
  it->graph_ff = ff->uid;
  it->graph_cons = cons_uid;
  it->graph_baro = baro_uid;
  it->graph_gen = ff->layout_gen;
  it->graph_thermo = thermo_uid;
  it->graph_pc = pc_uid;
  return HB_OK;
}

extern "C" int hb_integrator_step_graph(hb_integrator *it, hb_forcefield *ff,
                                        hb_constraints *cons, uint32_t n_steps) {
  HB_REQUIRE(it && ff, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_REQUIRE(ff->sys == it->sys && (!cons || cons->sys == it->sys), HB_ERR_INVALID_ARGUMENT,
             "integrator, force field and constraints must share one system");
  HB_TRY(lossless_prologue(it, cons));
  hb_context *ctx = it->sys->ctx;
  cudaStream_t s = ctx->stream;
  if (!it->forces_valid) {
    HB_TRY(force_eval(ff, false));
    it->forces_valid = true;
  }
  HB_TRY(ensure_step_graphs(it, ff, cons));
  if (ctx->timing) HB_CUDA(cudaEventRecord(it->g_ev0, s));
  for (uint32_t k = 0; k < n_steps; ++k) {
    const bool move = move_due(it, it->step + 1);
    HB_CUDA(cudaGraphLaunch(move ? it->graph_exec_move : it->graph_exec, s));
    it->step++;
  }
  if (ctx->timing) {
    HB_CUDA(cudaEventRecord(it->g_ev1, s));
    HB_CUDA(cudaEventSynchronize(it->g_ev1));
    float ms = 0.f;
    HB_CUDA(cudaEventElapsedTime(&ms, it->g_ev0, it->g_ev1));
    for (int q = 0; q < 8; ++q) ctx->t_ms[q] = 0.0;
    ctx->t_ms[0] = ms;
  }
  HB_TRY(check_status(ff));
  if (cons && cons->mlp) HB_TRY(mlp_status(cons->mlp));
  // buffers or sizes changed: the captured graphs are stale
  if (ff->layout_gen != it->graph_gen) drop_graphs(it);
  return HB_OK;
}

// ---- exchange steps: upload, steps and read-out in one call --------------
//
// Replaces the runner's "steps, then ParticleState::download_from" sequence
// (src/runner.rs:2709-2716, src/state.rs:140-216).  Positions and image
// counts are final once a step's head has run (kicks, drift, constraint
// projection), and so are the velocities of the Langevin middle scheme; the
// force evaluation only reads them.  Their conversion and device-to-host copy
// therefore run on a side stream concurrently with the force evaluation; the
// forces (and the velocity-Verlet velocities) follow the step's tail.  A step
// that ends with a volume move or scales positions in its tail (per-step
// pressure coupling) reads everything at its end.

struct ExchangeOut {
  float *pos, *vel, *force;
  int32_t *img;
};

// convert the requested fields into the output half of the staging buffer
// (the upload uses the first 6n floats) and copy them to the host arrays
static int readout_f32(hb_system *sys, cudaStream_t st, float *pos, float *vel, int32_t *img,
                       float *force) {
  if (!sys->n || (!pos && !vel && !img && !force)) return HB_OK;
  const size_t n = sys->n, n3 = 3 * n;
  float *base = reinterpret_cast<float *>(sys->d_stage);
  float *dp = base + 2 * n3, *dv = base + 3 * n3, *df = base + 4 * n3;
  k_state_out<float><<<hb_div_up(sys->n, 256), 256, 0, st>>>(
      sys->d_posq, sys->d_vel, sys->d_force, sys->d_image, pos ? dp : nullptr,
      vel ? dv : nullptr, force ? df : nullptr, img ? sys->d_stage_img : nullptr, sys->n);
  HB_CUDA(cudaGetLastError());
  if (pos) HB_CUDA(cudaMemcpyAsync(pos, dp, sizeof(float) * n3, cudaMemcpyDeviceToHost, st));
  if (vel) HB_CUDA(cudaMemcpyAsync(vel, dv, sizeof(float) * n3, cudaMemcpyDeviceToHost, st));
  if (force) HB_CUDA(cudaMemcpyAsync(force, df, sizeof(float) * n3, cudaMemcpyDeviceToHost, st));
  if (img)
    HB_CUDA(cudaMemcpyAsync(img, sys->d_stage_img, sizeof(int32_t) * n3, cudaMemcpyDeviceToHost,
                            st));
  return HB_OK;
}

// one step (with its volume move when `move`) whose state lands in `xo`
static int exchange_step(hb_integrator *it, hb_forcefield *ff, hb_constraints *cons, bool move,
                         bool capturing, const ExchangeOut &xo) {
  hb_system *sys = it->sys;
  hb_context *ctx = sys->ctx;
  cudaStream_t s = ctx->stream, sx = ctx->stream4;
  const bool early_pos = !move && (it->kind == HB_INTEGRATOR_LANGEVIN || !it->pc);
  const bool early_vel = !move && it->kind == HB_INTEGRATOR_LANGEVIN;
  ExchangeOut e{early_pos ? xo.pos : nullptr, early_vel ? xo.vel : nullptr, nullptr,
                early_pos ? xo.img : nullptr};
  const bool fork = e.pos || e.vel || e.img;
  HB_TRY(step_head(it, cons));
  if (fork) {
    HB_CUDA(cudaEventRecord(ctx->ev_xfork, s));
    HB_CUDA(cudaStreamWaitEvent(sx, ctx->ev_xfork, 0));
    HB_TRY(readout_f32(sys, sx, e.pos, e.vel, e.img, nullptr));
  }
  HB_TRY(force_eval(ff, step_force_ev(it, move), capturing));
  HB_TRY(step_tail(it, ff, cons));
  if (move) HB_TRY(baro_move(it->baro, ff, capturing));
  HB_TRY(readout_f32(sys, s, e.pos ? nullptr : xo.pos, e.vel ? nullptr : xo.vel,
                     e.img ? nullptr : xo.img, xo.force));
  if (fork) {
    HB_CUDA(cudaEventRecord(ctx->ev_xjoin, sx));
    HB_CUDA(cudaStreamWaitEvent(s, ctx->ev_xjoin, 0));
  }
  return HB_OK;
}

static int capture_exchange(hb_integrator *it, hb_forcefield *ff, hb_constraints *cons, bool move,
                            const ExchangeOut &xo, cudaGraphExec_t *exec) {
  cudaStream_t s = it->sys->ctx->stream;
  cudaGraph_t g;
  HB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const uint64_t step = it->step;
  int rc = exchange_step(it, ff, cons, move, true, xo);
  it->step = step;
  cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (rc != HB_OK) return rc;
  if (ce != cudaSuccess) return hb_fail(HB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
  cudaError_t ie = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) return hb_fail(HB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
  return HB_OK;
}

static bool page_locked(const void *p) {
  if (!p) return true;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

extern "C" int hb_integrator_step_exchange_f32(hb_integrator *it, hb_forcefield *ff,
                                               hb_constraints *cons, uint32_t n_steps,
                                               const float *positions_in,
                                               const float *velocities_in, float *positions,
                                               float *velocities, int32_t *images,
                                               float *forces) {
  HB_REQUIRE(it && ff, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_REQUIRE(ff->sys == it->sys && (!cons || cons->sys == it->sys), HB_ERR_INVALID_ARGUMENT,
             "integrator, force field and constraints must share one system");
  HB_REQUIRE(n_steps >= 1, HB_ERR_INVALID_ARGUMENT, "an exchange call takes at least one step");
  hb_system *sys = it->sys;
  HB_TRY(set_state_t<float>(sys, positions_in, velocities_in));
  const ExchangeOut xo{positions, velocities, forces, images};
  if (!page_locked(positions) || !page_locked(velocities) || !page_locked(forces) ||
      !page_locked(images)) {
    // pageable host arrays cannot be graph copy targets: steps, then read-out
    HB_TRY(hb_integrator_step_graph(it, ff, cons, n_steps));
    return get_state_t<float>(sys, positions, velocities, images, forces);
  }
  HB_TRY(lossless_prologue(it, cons));
  hb_context *ctx = sys->ctx;
  cudaStream_t s = ctx->stream;
  if (!it->forces_valid) {
    HB_TRY(force_eval(ff, false));
    it->forces_valid = true;
  }
  HB_TRY(stage_alloc(sys));
  HB_TRY(ensure_step_graphs(it, ff, cons));
  const void *key[4] = {positions, velocities, forces, images};
  if (!std::equal(key, key + 4, it->graph_x_key)) {
    drop_exchange_graphs(it);
    HB_CUDA(cudaStreamSynchronize(s));
    HB_TRY(capture_exchange(it, ff, cons, false, xo, &it->graph_exec_x));
    if (it->baro) HB_TRY(capture_exchange(it, ff, cons, true, xo, &it->graph_exec_x_move));
    std::copy(key, key + 4, it->graph_x_key);
  }
  if (ctx->timing) HB_CUDA(cudaEventRecord(it->g_ev0, s));
  for (uint32_t k = 0; k < n_steps; ++k) {
    const bool move = move_due(it, it->step + 1);
    cudaGraphExec_t g = k + 1 < n_steps ? (move ? it->graph_exec_move : it->graph_exec)
                                        : (move ? it->graph_exec_x_move : it->graph_exec_x);
    HB_CUDA(cudaGraphLaunch(g, s));
    it->step++;
  }
  if (ctx->timing) {
    HB_CUDA(cudaEventRecord(it->g_ev1, s));
    HB_CUDA(cudaEventSynchronize(it->g_ev1));
    float ms = 0.f;
    HB_CUDA(cudaEventElapsedTime(&ms, it->g_ev0, it->g_ev1));
    for (int q = 0; q < 8; ++q) ctx->t_ms[q] = 0.0;
    ctx->t_ms[0] = ms;
  }
  // check_status synchronises the stream: the host arrays are filled
  HB_TRY(check_status(ff));
  if (cons && cons->mlp) HB_TRY(mlp_status(cons->mlp));
  if (ff->layout_gen != it->graph_gen) drop_graphs(it);
  return HB_OK;
}

static int count_kernel_nodes(cudaGraph_t g, uint64_t &kernels) {
  size_t nn = 0;
  HB_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn) HB_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    HB_CUDA(cudaGraphNodeGetType(nd, &t));
    if (t == cudaGraphNodeTypeKernel) ++kernels;
  }
  return HB_OK;
}

static int count_captured(hb_integrator *it, hb_forcefield *ff, hb_constraints *cons, bool step,
                          bool move, uint64_t &kernels) {
  cudaStream_t s = it->sys->ctx->stream;
  cudaGraph_t g;
  HB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const uint64_t st = it->step;
  int rc = step ? one_step(it, ff, cons, false, false) : HB_OK;
  if (rc == HB_OK && move) rc = baro_move(it->baro, ff, false);
  it->step = st;
  cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (rc != HB_OK) return rc;
  if (ce != cudaSuccess) return hb_fail(HB_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
  kernels = 0;
  rc = count_kernel_nodes(g, kernels);
  cudaGraphDestroy(g);
  return rc;
}

extern "C" int hb_integrator_count_launches(hb_integrator *it, hb_forcefield *ff,
                                            hb_constraints *cons, uint64_t *kernels) {
  HB_REQUIRE(it && ff && kernels, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_CUDA(cudaStreamSynchronize(it->sys->ctx->stream));
  // capture the eager launch sequence (rebuild kernels gated, no
  // conditional node) and count its kernel nodes; nothing runs
  uint64_t eager = 0, eager_move = 0;
  HB_TRY(count_captured(it, ff, cons, true, false, eager));
  if (it->baro && it->sys->n) HB_TRY(count_captured(it, ff, cons, false, true, eager_move));
  // in the graph form the gated rebuild kernels move into the IF node's
  // body and one kernel sets the condition
  const uint64_t body = ff->sys->n ? (uint64_t)nl_kernel_count() : 0u;
  kernels[0] = eager - body + (body ? 1u : 0u);
  kernels[1] = body;
  kernels[2] = eager_move ? eager_move - body + 1u : 0u;
  return HB_OK;
}

// ---------------------------------------------------------------------
// batched replicas
// ---------------------------------------------------------------------
struct hb_batch {
  hb_context *ctx = nullptr;                 // the graph launches on its stream
  std::vector<hb_integrator *> its;
  std::vector<hb_forcefield *> ffs;
  std::vector<hb_constraints *> cons;
  std::vector<cudaEvent_t> join;             // one per member
  std::vector<cudaEvent_t> ready;            // a member's step up to its pair kernel
  std::vector<uint64_t> gens;                // members' layout_gen at capture
  cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr, pair_done = nullptr;
  cudaGraphExec_t exec = nullptr;
  // 1: one multi-system pair launch for all members (when they share the
  // pair physics and contexts are distinct); 0 (default, measured faster:
  // members that skip a rebuild start their pair kernels early instead of
  // waiting at the join) = one pair launch per member
  int one_pair_launch = 0;
  bool multi = false;                        // the form of the captured graph
  void *d_members = nullptr;                 // member table of the multi-system launch
  uint32_t *d_work = nullptr;                // its work counter
  uint32_t items = 0;
};

extern "C" int hb_batch_destroy(hb_batch *b) {
  if (!b) return HB_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (auto e : b->join)
    if (e) cudaEventDestroy(e);
  for (auto e : b->ready)
    if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->t0) cudaEventDestroy(b->t0);
  if (b->t1) cudaEventDestroy(b->t1);
  if (b->pair_done) cudaEventDestroy(b->pair_done);
  cudaFree(b->d_members);
  cudaFree(b->d_work);
  delete b;
  return HB_OK;
}

extern "C" int hb_batch_create(hb_context *ctx, uint32_t n, hb_integrator *const *its,
                               hb_forcefield *const *ffs, hb_constraints *const *cons,
                               hb_batch **out) {
  HB_REQUIRE(ctx && its && ffs && out && n > 0, HB_ERR_INVALID_ARGUMENT, "null argument");
  for (uint32_t k = 0; k < n; ++k) {
    HB_REQUIRE(its[k] && ffs[k], HB_ERR_INVALID_ARGUMENT, "null batch member");
    HB_REQUIRE(ffs[k]->sys == its[k]->sys && (!cons || !cons[k] || cons[k]->sys == its[k]->sys),
               HB_ERR_INVALID_ARGUMENT, "a member's integrator, force field and constraints "
                                        "must share one system");
    HB_REQUIRE(its[k]->sys->ctx->device == ctx->device, HB_ERR_INVALID_ARGUMENT,
               "batch members must live on the batch's device");
    HB_REQUIRE(its[k]->sys->ctx != ctx, HB_ERR_INVALID_ARGUMENT,
               "batch members need contexts of their own (the batch context launches the graph)");
    HB_REQUIRE(!its[k]->baro, HB_ERR_UNSUPPORTED, "batch members take no barostat");
    for (uint32_t q = 0; q < k; ++q)
      HB_REQUIRE(its[q]->sys != its[k]->sys, HB_ERR_INVALID_ARGUMENT,
                 "a system may appear in one batch member only");
  }
  hb_batch *b = new hb_batch();
  b->ctx = ctx;
  b->its.assign(its, its + n);
  b->ffs.assign(ffs, ffs + n);
  b->cons.assign(n, nullptr);
  if (cons)
    for (uint32_t k = 0; k < n; ++k) b->cons[k] = cons[k];
  b->join.assign(n, nullptr);
  b->ready.assign(n, nullptr);
  bool ok = cudaSetDevice(ctx->device) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->pair_done, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreate(&b->t0) == cudaSuccess && cudaEventCreate(&b->t1) == cudaSuccess &&
            cudaMalloc(&b->d_members, pair_member_bytes() * n) == cudaSuccess &&
            cudaMalloc(&b->d_work, sizeof(uint32_t)) == cudaSuccess;
  for (uint32_t k = 0; ok && k < n; ++k)
    ok = cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&b->ready[k], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    hb_batch_destroy(b);
    return hb_fail(HB_ERR_CUDA, "batch event creation failed");
  }
  *out = b;
  return HB_OK;
}

// whether the members' pair kernels can run as one multi-system launch:
// the same pair physics, force-only steps (no per-step pressure coupling),
// and a context (streams, events) of their own each
static bool batch_multi_ok(const hb_batch *b) {
  if (!b->one_pair_launch) return false;
  const size_t n = b->its.size();
  for (size_t k = 0; k < n; ++k) {
    if (step_force_ev(b->its[k], false)) return false;
    for (size_t q = 0; q < k; ++q)
      if (b->its[q]->sys->ctx == b->its[k]->sys->ctx) return false;
  }
  return pair_batchable(b->ffs.data(), (uint32_t)n);
}

// one graph: fork from the batch stream to every member's stream and
// capture the member's step there, join back.  In the multi-system form
// each member runs up to its pair kernel, the batch stream waits for all
// of them and launches one pair kernel over every member's work items, and
// each member then finishes its step (reciprocal-space join, finalize,
// final kick) after that launch.
static int batch_capture(hb_batch *b) {
  const size_t n = b->its.size();
  b->multi = batch_multi_ok(b);
  if (b->multi) HB_TRY(pair_batch_table(b->ffs.data(), (uint32_t)n, b->d_members, &b->items));
  cudaStream_t m = b->ctx->stream;
  cudaGraph_t g;
  HB_CUDA(cudaStreamBeginCapture(m, cudaStreamCaptureModeThreadLocal));
  int rc = cudaEventRecord(b->fork, m) == cudaSuccess ? HB_OK : HB_ERR_CUDA;
  std::vector<uint64_t> steps(n);
  for (size_t k = 0; k < n && rc == HB_OK; ++k) {
    hb_integrator *it = b->its[k];
    cudaStream_t s = it->sys->ctx->stream;
    if (cudaStreamWaitEvent(s, b->fork, 0) != cudaSuccess) {
      rc = hb_fail(HB_ERR_CUDA, "batch fork");
      break;
    }
    steps[k] = it->step;
    if (!b->multi) {
      rc = one_step(it, b->ffs[k], b->cons[k], false, true);
      it->step = steps[k];
      if (rc == HB_OK && (cudaEventRecord(b->join[k], s) != cudaSuccess ||
                          cudaStreamWaitEvent(m, b->join[k], 0) != cudaSuccess))
        rc = hb_fail(HB_ERR_CUDA, "batch join");
      continue;
    }
    rc = step_head(it, b->cons[k]);
    if (rc == HB_OK) rc = force_pre(b->ffs[k], false, true);
    if (rc == HB_OK && (cudaEventRecord(b->ready[k], s) != cudaSuccess ||
                        cudaStreamWaitEvent(m, b->ready[k], 0) != cudaSuccess))
      rc = hb_fail(HB_ERR_CUDA, "batch join");
  }
  if (b->multi && rc == HB_OK) {
    rc = pair_launch_batch(b->ffs.data(), (uint32_t)n, b->d_members, b->items, b->d_work, m);
    if (rc == HB_OK && cudaEventRecord(b->pair_done, m) != cudaSuccess)
      rc = hb_fail(HB_ERR_CUDA, "batch pair launch");
    for (size_t k = 0; k < n && rc == HB_OK; ++k) {
      hb_integrator *it = b->its[k];
      cudaStream_t s = it->sys->ctx->stream;
      if (cudaStreamWaitEvent(s, b->pair_done, 0) != cudaSuccess) {
        rc = hb_fail(HB_ERR_CUDA, "batch fork");
        break;
      }
      rc = force_post(b->ffs[k], false);
      if (rc == HB_OK) rc = step_tail(it, b->ffs[k], b->cons[k]);
      it->step = steps[k];
      if (rc == HB_OK && (cudaEventRecord(b->join[k], s) != cudaSuccess ||
                          cudaStreamWaitEvent(m, b->join[k], 0) != cudaSuccess))
        rc = hb_fail(HB_ERR_CUDA, "batch join");
    }
  }
  cudaError_t ce = cudaStreamEndCapture(m, &g);
  if (rc != HB_OK) return rc;
  if (ce != cudaSuccess) return hb_fail(HB_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(ce));
  cudaError_t ie = cudaGraphInstantiate(&b->exec, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) return hb_fail(HB_ERR_CUDA, std::string("batch instantiate: ") + cudaGetErrorString(ie));
  return HB_OK;
}

extern "C" int hb_batch_set_pair_form(hb_batch *b, int one_launch) {
  HB_REQUIRE(b, HB_ERR_INVALID_ARGUMENT, "null batch");
  b->one_pair_launch = one_launch ? 1 : 0;
  if (b->exec) {
    cudaStreamSynchronize(b->ctx->stream);
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  return HB_OK;
}

extern "C" int hb_batch_pair_form(hb_batch *b, int *one_launch) {
  HB_REQUIRE(b && one_launch, HB_ERR_INVALID_ARGUMENT, "null argument");
  *one_launch = batch_multi_ok(b) ? 1 : 0;
  return HB_OK;
}

extern "C" int hb_batch_step(hb_batch *b, uint32_t n_steps) {
  HB_REQUIRE(b, HB_ERR_INVALID_ARGUMENT, "null batch");
  hb_context *ctx = b->ctx;
  const size_t n = b->its.size();
  for (size_t k = 0; k < n; ++k) {
    hb_integrator *it = b->its[k];
    HB_REQUIRE(!it->baro, HB_ERR_UNSUPPORTED, "batch members take no barostat");
    HB_TRY(lossless_prologue(it, b->cons[k]));
    if (!it->forces_valid) {
      HB_TRY(force_eval(b->ffs[k], false));
      it->forces_valid = true;
    }
  }
  // member streams before the batch stream: eager work above, then the graph
  for (size_t k = 0; k < n; ++k) HB_CUDA(cudaStreamSynchronize(b->its[k]->sys->ctx->stream));
  bool stale = b->gens.size() != n;
  for (size_t k = 0; k < n && !stale; ++k) stale = b->gens[k] != b->ffs[k]->layout_gen;
  if (stale && b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (!b->exec) {
    HB_TRY(batch_capture(b));
    b->gens.resize(n);
    for (size_t k = 0; k < n; ++k) b->gens[k] = b->ffs[k]->layout_gen;
  }
  cudaStream_t m = ctx->stream;
  if (ctx->timing) HB_CUDA(cudaEventRecord(b->t0, m));
  for (uint32_t q = 0; q < n_steps; ++q) {
    HB_CUDA(cudaGraphLaunch(b->exec, m));
    for (size_t k = 0; k < n; ++k) b->its[k]->step++;
  }
  if (ctx->timing) HB_CUDA(cudaEventRecord(b->t1, m));
  HB_CUDA(cudaStreamSynchronize(m));
  if (ctx->timing) {
    float ms = 0.f;
    HB_CUDA(cudaEventElapsedTime(&ms, b->t0, b->t1));
    for (int q = 0; q < 8; ++q) ctx->t_ms[q] = 0.0;
    ctx->t_ms[0] = ms;
  }
  // a member whose list grows bumps its layout_gen: the next call recaptures
  for (size_t k = 0; k < n; ++k) HB_TRY(check_status(b->ffs[k]));
  return HB_OK;
}

extern "C" int hb_batch_count_launches(hb_batch *b, uint64_t kernels[2]) {
  HB_REQUIRE(b && kernels, HB_ERR_INVALID_ARGUMENT, "null argument");
  kernels[0] = kernels[1] = 0;
  for (size_t k = 0; k < b->its.size(); ++k) {
    uint64_t c[3] = {0, 0, 0};
    HB_TRY(hb_integrator_count_launches(b->its[k], b->ffs[k], b->cons[k], c));
    kernels[0] += c[0];
    kernels[1] += c[1];
  }
  // the multi-system form: one pair kernel for all members
  if (batch_multi_ok(b)) kernels[0] -= (uint64_t)(b->its.size() - 1);
  return HB_OK;
}

extern "C" int hb_reduce_kinetic(hb_system *sys, double out[4]) {
  HB_REQUIRE(sys && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  return reduce_kinetic(sys, out);
}

extern "C" int hb_timing_enable(hb_context *ctx, int enable) {
  HB_REQUIRE(ctx, HB_ERR_INVALID_ARGUMENT, "null context");
  ctx->timing = enable != 0;
  return HB_OK;
}

extern "C" int hb_timing_get(hb_context *ctx, double out[8]) {
  HB_REQUIRE(ctx && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  for (int q = 0; q < 8; ++q) out[q] = ctx->t_ms[q];
  return HB_OK;
}
