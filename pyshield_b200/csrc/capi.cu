// C-ABI entry points of libshield_mp.so (declared in include/shield_mp.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/shield_mp.h"
#include "mp_launch.h"
#include "mp_params.h"
#include "mp_setup.h"

using namespace shield;

namespace {

thread_local std::string g_last_error;

struct Handle {
  ShieldMpConfig cfg;
  int nx, ny, nz;
  int64_t ncol;
  int device;
  double* area = nullptr;  // device copy of grid_data.area (ncol)
  double* qaz = nullptr;   // persistent accumulator, nz * ncol, level-major
  int* err = nullptr;
  double* vjp_ws = nullptr;  // the adjoint's workspace, allocated by its first call and grown as needed
  int64_t vjp_ws_doubles = 0;
  MpConst K;
  bool have_ts = false;
  std::string last_error;
};

int fail(Handle* h, int code, const std::string& msg) {
  if (h) h->last_error = msg;
  g_last_error = msg;
  return code;
}

int cuda_fail(Handle* h, cudaError_t e, const char* what) {
  return fail(h, SHIELD_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

Fld3 f3(const ShieldField3D& f) { return Fld3{f.ptr, f.si, f.sj, f.sk}; }

}  // namespace

namespace shield {
// The handle-free calls (coupling kernels) report through here.
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace shield

extern "C" int shield_mp_create(const ShieldMpConfig* cfg, int nx, int ny, int nz, ShieldField2D area,
                                void** handle) {
  if (!cfg || !handle) return fail(nullptr, SHIELD_EINVAL, "null config or handle pointer");
  *handle = nullptr;
  if (nx < 1 || ny < 1) return fail(nullptr, SHIELD_EINVAL, "nx and ny must be positive");
  if (nz < 3 || nz > mp_max_levels()) return fail(nullptr, SHIELD_ELAYOUT, "nz must lie in [3, 256]");
  if (cfg->use_ppm) return fail(nullptr, SHIELD_EINVAL, "use_ppm=True is not supported (incomplete in the reference)");
  if (!area.ptr) return fail(nullptr, SHIELD_EINVAL, "null area pointer");
  Handle* h = new Handle();
  h->cfg = *cfg;
  h->nx = nx;
  h->ny = ny;
  h->nz = nz;
  h->ncol = (int64_t)nx * ny;
  cudaError_t e = cudaGetDevice(&h->device);
  if (e != cudaSuccess) {
    int rc = cuda_fail(h, e, "cudaGetDevice");
    delete h;
    return rc;
  }
  setupm(*cfg, h->K);
  std::string why;
  if (set_timestep(*cfg, h->K, cfg->dt_atmos, why) != SHIELD_OK) {
    delete h;
    return fail(nullptr, SHIELD_EINVAL, "dt_atmos: " + why);
  }
  h->have_ts = true;
  const size_t qbytes = sizeof(double) * (size_t)h->ncol * nz;
  if ((e = cudaMalloc(&h->qaz, qbytes)) != cudaSuccess || (e = cudaMemset(h->qaz, 0, qbytes)) != cudaSuccess ||
      (e = cudaMalloc(&h->area, sizeof(double) * h->ncol)) != cudaSuccess ||
      (e = cudaMalloc(&h->err, sizeof(int))) != cudaSuccess || (e = cudaMemset(h->err, 0, sizeof(int))) != cudaSuccess) {
    int rc = cuda_fail(nullptr, e, "allocating handle state");
    cudaFree(h->qaz);
    cudaFree(h->area);
    cudaFree(h->err);
    delete h;
    return rc;
  }
  e = mp_gather_area(area.ptr, area.si, area.sj, nx, ny, h->area);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    int rc = cuda_fail(nullptr, e, "copying area");
    cudaFree(h->qaz);
    cudaFree(h->area);
    cudaFree(h->err);
    delete h;
    return rc;
  }
  *handle = h;
  return SHIELD_OK;
}

namespace {

// The step of shield_mp_step; with `flags` non-null (plain form only) the
// launch also records each sub-step's column flags there.
int step_impl(Handle* h, const ShieldMpFields* F, double timestep, int precision, int32_t* flags, int64_t nflags,
              void* stream) {
  if (!h) return fail(nullptr, SHIELD_EINVAL, "null handle");
  if (!F) return fail(h, SHIELD_EINVAL, "null fields");
  if (precision != SHIELD_MP_PLAIN && precision != SHIELD_MP_MIXED)
    return fail(h, SHIELD_EINVAL, "unknown precision mode");
  if (timestep != h->K.timestep) {
    std::string why;
    MpConst K2 = h->K;
    if (set_timestep(h->cfg, K2, timestep, why) != SHIELD_OK) return fail(h, SHIELD_EINVAL, why);
    h->K = K2;
  }
  const ShieldField3D* ins[] = {&F->pt, &F->qvapor, &F->qliquid, &F->qrain, &F->qice, &F->qsnow, &F->qgraupel,
                                &F->qcld, &F->ua, &F->va, &F->delprsi, &F->delz, &F->wmp};
  const ShieldField3D* outs[] = {&F->pt_dt, &F->qv_dt, &F->ql_dt, &F->qr_dt, &F->qi_dt,
                                 &F->qs_dt, &F->qg_dt, &F->qa_dt, &F->udt,   &F->vdt};
  MpArgs A;
  std::memset(&A, 0, sizeof(A));
  A.K = h->K;
  A.KF = to_float(h->K);
  A.nx = h->nx;
  A.ny = h->ny;
  A.nz = h->nz;
  A.ncol = h->ncol;
  for (int f = 0; f < 13; ++f) {
    if (!ins[f]->ptr) return fail(h, SHIELD_EINVAL, "null input field pointer");
    A.in[f] = f3(*ins[f]);
  }
  const Fld3 qaz{h->qaz, 1, h->nx, h->ncol};
  A.in[IN_QAZ] = qaz;
  for (int o = 0; o < 10; ++o) {
    if (!outs[o]->ptr) return fail(h, SHIELD_EINVAL, "null tendency pointer");
    A.out[o] = f3(*outs[o]);
  }
  A.out[OUT_W] = A.in[IN_W];
  A.out[OUT_QAZ] = qaz;
  if (!F->land.ptr) return fail(h, SHIELD_EINVAL, "null land pointer");
  A.land = Fld2{F->land.ptr, F->land.si, F->land.sj};
  A.area = Fld2{h->area, 1, h->nx};
  A.rain = F->rain;
  A.snow = F->snow;
  A.ice = F->ice;
  A.graupel = F->graupel;
  A.err = h->err;
  if (flags) {
    if (precision != SHIELD_MP_PLAIN) return fail(h, SHIELD_EINVAL, "column flags are recorded by the plain form only");
    if (nflags < (int64_t)h->K.ntimes * h->ncol)
      return fail(h, SHIELD_EINVAL,
                  "the flags buffer holds " + std::to_string(nflags) + " words; this step needs ntimes * nx * ny = " +
                      std::to_string((int64_t)h->K.ntimes * h->ncol));
    A.flags = flags;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaSuccess;
  if (h->K.de_ice) {
    e = mp_launch_de_ice(A, f3(F->qi_dt), f3(F->qs_dt), st);
    if (e != cudaSuccess) return cuda_fail(h, e, "de_ice launch");
  }
  e = flags ? mp_launch_plain_flags(A, st) : mp_launch_step(A, precision, st);
  if (e != cudaSuccess) return cuda_fail(h, e, "microphysics launch");
  return SHIELD_OK;
}

}  // namespace

extern "C" int shield_mp_step(void* handle, const ShieldMpFields* F, double timestep, int precision, void* stream) {
  return step_impl(static_cast<Handle*>(handle), F, timestep, precision, nullptr, 0, stream);
}

extern "C" int shield_mp_step_flags(void* handle, const ShieldMpFields* F, double timestep, int32_t* flags,
                                    int64_t nflags, void* stream) {
  if (!flags) return fail(static_cast<Handle*>(handle), SHIELD_EINVAL, "null flags buffer");
  return step_impl(static_cast<Handle*>(handle), F, timestep, SHIELD_MP_PLAIN, flags, nflags, stream);
}

extern "C" int shield_mp_substeps(void* handle, double timestep) {
  Handle* h = static_cast<Handle*>(handle);
  if (!h) return fail(nullptr, SHIELD_EINVAL, "null handle");
  MpConst K2 = h->K;
  std::string why;
  if (set_timestep(h->cfg, K2, timestep, why) != SHIELD_OK) return fail(h, SHIELD_EINVAL, why);
  return K2.ntimes;
}

extern "C" int shield_mp_step_vjp(void* handle, const ShieldMpFields* F, const ShieldMpCotangents* cot,
                                  const ShieldMpGradients* grad, double timestep, void* stream) {
  Handle* h = static_cast<Handle*>(handle);
  if (!h) return fail(nullptr, SHIELD_EINVAL, "null handle");
  if (!F || !cot || !grad) return fail(h, SHIELD_EINVAL, "null fields, cotangents or gradients");
  MpConst K = h->K;
  if (timestep != K.timestep) {
    std::string why;
    if (set_timestep(h->cfg, K, timestep, why) != SHIELD_OK) return fail(h, SHIELD_EINVAL, why);
  }
  const int64_t need = mp_vjp_workspace_doubles(K.ntimes, (int64_t)h->nz * h->ncol, h->ncol);
  if (need > h->vjp_ws_doubles) {
    cudaFree(h->vjp_ws);
    h->vjp_ws = nullptr;
    h->vjp_ws_doubles = 0;
    cudaError_t e = cudaMalloc(&h->vjp_ws, sizeof(double) * (size_t)need);
    if (e != cudaSuccess) {
      h->vjp_ws = nullptr;
      return cuda_fail(h, e, "allocating the adjoint's workspace");
    }
    h->vjp_ws_doubles = need;
  }
  VjpArgs A;
  std::memset(&A, 0, sizeof(A));
  A.K = K;
  A.KF = to_float(K);
  A.nx = h->nx;
  A.ny = h->ny;
  A.nz = h->nz;
  A.ncol = h->ncol;
  const ShieldField3D* ins[] = {&F->pt, &F->qvapor, &F->qliquid, &F->qrain, &F->qice, &F->qsnow, &F->qgraupel,
                                &F->qcld, &F->ua, &F->va, &F->delprsi, &F->delz, &F->wmp};
  const ShieldField3D* cots[] = {&cot->pt_dt, &cot->qv_dt, &cot->ql_dt, &cot->qr_dt, &cot->qi_dt, &cot->qs_dt,
                                 &cot->qg_dt, &cot->qa_dt, &cot->udt,   &cot->vdt,   &cot->wmp,   &cot->qaz};
  const ShieldField3D* grads[] = {&grad->pt,   &grad->qvapor, &grad->qliquid, &grad->qrain, &grad->qice,
                                  &grad->qsnow, &grad->qgraupel, &grad->qcld,  &grad->ua,    &grad->va,
                                  &grad->delprsi, &grad->delz,  &grad->wmp,   &grad->qaz};
  for (int f = 0; f < N_VJP_IN; ++f) {
    if (!ins[f]->ptr) return fail(h, SHIELD_EINVAL, "null input field pointer");
    A.in[f] = f3(*ins[f]);
  }
  for (int f = 0; f < N_VJP_COT; ++f) A.cot[f] = f3(*cots[f]);
  for (int f = 0; f < N_VJP_GRAD; ++f) A.grad[f] = f3(*grads[f]);
  if (!F->land.ptr) return fail(h, SHIELD_EINVAL, "null land pointer");
  A.land = Fld2{F->land.ptr, F->land.si, F->land.sj};
  A.area = Fld2{h->area, 1, h->nx};
  A.rain_b = cot->rain;
  A.snow_b = cot->snow;
  A.ice_b = cot->ice;
  A.graupel_b = cot->graupel;
  A.ws = h->vjp_ws;
  A.de_ice_qi_dt = f3(F->qi_dt);
  cudaError_t e = mp_launch_vjp(A, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(h, e, "adjoint launch");
  return SHIELD_OK;
}

// The device error word of the handle's steps: which column, if any,
// produced a NaN or an infinity since the last check. Waits for `stream`.
extern "C" int shield_mp_check(void* handle, int64_t* bad_column, void* stream) {
  Handle* h = static_cast<Handle*>(handle);
  if (!h) return fail(nullptr, SHIELD_EINVAL, "null handle");
  if (bad_column) *bad_column = -1;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(h, e, "reading the error word");
  if (v == 0) return SHIELD_OK;
  e = cudaMemsetAsync(h->err, 0, sizeof(int), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(h, e, "clearing the error word");
  const int64_t c = (int64_t)v - 1;
  if (bad_column) *bad_column = c;
  return fail(h, SHIELD_EDEVICE,
              "column " + std::to_string(c) + " (i = " + std::to_string(c % h->nx) + ", j = " +
                  std::to_string(c / h->nx) + ") produced a NaN or an infinity");
}

extern "C" int shield_mp_destroy(void* handle) {
  Handle* h = static_cast<Handle*>(handle);
  if (!h) return SHIELD_OK;
  cudaFree(h->qaz);
  cudaFree(h->area);
  cudaFree(h->err);
  cudaFree(h->vjp_ws);
  delete h;
  return SHIELD_OK;
}

extern "C" int shield_mp_last_error(void* handle, char* buf, size_t n) {
  Handle* h = static_cast<Handle*>(handle);
  const std::string& m = h ? h->last_error : g_last_error;
  if (buf && n) {
    std::strncpy(buf, m.c_str(), n - 1);
    buf[n - 1] = 0;
  }
  return SHIELD_OK;
}

extern "C" int shield_last_error(char* buf, size_t n) {
  if (buf && n) {
    std::strncpy(buf, g_last_error.c_str(), n - 1);
    buf[n - 1] = 0;
  }
  return SHIELD_OK;
}

extern "C" int shield_mp_constants(void* handle, double timestep, double* out, int n) {
  Handle* h = static_cast<Handle*>(handle);
  if (!h || !out) return SHIELD_EINVAL;
  MpConst K = h->K;
  std::string why;
  if (set_timestep(h->cfg, K, timestep, why) != SHIELD_OK) return fail(h, SHIELD_EINVAL, why);
  const double* src = reinterpret_cast<const double*>(&K);
  // the leading block of doubles, up to the first int member (ntimes)
  const int nd = (int)(offsetof(MpConst, ntimes) / sizeof(double));
  const int m = n < nd ? n : nd;
  std::memcpy(out, src, sizeof(double) * m);
  return m;
}

extern "C" int shield_mp_setup_constants(const ShieldMpConfig* cfg, double timestep, double* out, int n) {
  if (!cfg || !out) return fail(nullptr, SHIELD_EINVAL, "null argument");
  MpConst K;
  std::memset(&K, 0, sizeof(K));
  setupm(*cfg, K);
  std::string why;
  if (set_timestep(*cfg, K, timestep, why) != SHIELD_OK) return fail(nullptr, SHIELD_EINVAL, why);
  const double* src = reinterpret_cast<const double*>(&K);
  const int nd = (int)(offsetof(MpConst, ntimes) / sizeof(double));
  const int m = n < nd ? n : nd;
  std::memcpy(out, src, sizeof(double) * m);
  return m;
}

extern "C" int shield_mp_get_qaz(void* handle, double* qaz, void* stream) {
  Handle* h = static_cast<Handle*>(handle);
  if (!h || !qaz) return fail(h, SHIELD_EINVAL, "null argument");
  cudaError_t e = cudaMemcpyAsync(qaz, h->qaz, sizeof(double) * h->ncol * h->nz, cudaMemcpyDeviceToDevice,
                                  static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? SHIELD_OK : cuda_fail(h, e, "copying qaz");
}

extern "C" int shield_mp_set_qaz(void* handle, const double* qaz, void* stream) {
  Handle* h = static_cast<Handle*>(handle);
  if (!h || !qaz) return fail(h, SHIELD_EINVAL, "null argument");
  cudaError_t e = cudaMemcpyAsync(h->qaz, qaz, sizeof(double) * h->ncol * h->nz, cudaMemcpyDeviceToDevice,
                                  static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? SHIELD_OK : cuda_fail(h, e, "copying qaz");
}

// ------------------------------------------------------------------ ensembles
namespace {

struct Plan {
  int nm = 0, nz = 0, precision = 0, num_sms = 0;
  MpArgs* d_members = nullptr;
  int64_t* d_offs[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // cols_per_block 1, 2, 4, 6, 8
  double* d_area = nullptr;
  double* d_qaz = nullptr;
  unsigned long long* d_counter = nullptr;  // the launch's work-item counter
  std::vector<int64_t> qaz_off;
  int64_t qaz_total = 0;
  std::string last_error;
};

int gindex(int G) { return G == 1 ? 0 : G == 2 ? 1 : G == 4 ? 2 : G == 6 ? 3 : G == 8 ? 4 : -1; }

// cols_per_block values the ensemble launch has for nz levels: 65..80 levels
// pack two columns per 5 warps, so a block holds 2, 4, 6 or 8 columns.
bool ensemble_shape_ok(int nz, int G) {
  if (nz <= 80) return G == 2 || G == 4 || G == 6 || G == 8;
  return G == 1 || G == 2 || G == 4;
}

void plan_free(Plan* p) {
  cudaFree(p->d_members);
  for (auto& o : p->d_offs) cudaFree(o);
  cudaFree(p->d_area);
  cudaFree(p->d_qaz);
  cudaFree(p->d_counter);
  delete p;
}

}  // namespace

extern "C" int shield_mp_ensemble_create(const ShieldMpConfig* cfg, int nz, int nm, const ShieldMpMember* mem,
                                         int precision, void** plan) {
  if (!cfg || !mem || !plan || nm < 1) return fail(nullptr, SHIELD_EINVAL, "bad ensemble arguments");
  *plan = nullptr;
  if (nz <= 64 || nz > 128) return fail(nullptr, SHIELD_ELAYOUT, "ensembles support 65..128 levels");
  if (precision != SHIELD_MP_PLAIN && precision != SHIELD_MP_MIXED) return fail(nullptr, SHIELD_EINVAL, "precision");
  if (cfg->use_ppm) return fail(nullptr, SHIELD_EINVAL, "use_ppm=True is not supported");
  Plan* p = new Plan();
  p->nm = nm;
  p->nz = nz;
  p->precision = precision;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) {
    int rc = cuda_fail(nullptr, e, "device query");
    plan_free(p);
    return rc;
  }
  std::vector<MpArgs> host(nm);
  int64_t area_total = 0, qaz_total = 0;
  std::vector<int64_t> area_off(nm);
  p->qaz_off.resize(nm);
  MpConst base;
  std::memset(&base, 0, sizeof(base));
  setupm(*cfg, base);
  for (int m = 0; m < nm; ++m) {
    const ShieldMpMember& M = mem[m];
    if (M.nx < 1 || M.ny < 1 || !M.area.ptr) {
      plan_free(p);
      return fail(nullptr, SHIELD_EINVAL, "member " + std::to_string(m) + ": bad domain or area");
    }
    MpArgs& A = host[m];
    std::memset(&A, 0, sizeof(A));
    A.K = base;
    std::string why;
    if (set_timestep(*cfg, A.K, M.timestep, why) != SHIELD_OK) {
      plan_free(p);
      return fail(nullptr, SHIELD_EINVAL, "member " + std::to_string(m) + ": " + why);
    }
    A.KF = to_float(A.K);
    A.nx = M.nx;
    A.ny = M.ny;
    A.nz = nz;
    A.ncol = (int64_t)M.nx * M.ny;
    const ShieldMpFields& F = M.fields;
    const ShieldField3D* ins[] = {&F.pt, &F.qvapor, &F.qliquid, &F.qrain, &F.qice, &F.qsnow, &F.qgraupel,
                                  &F.qcld, &F.ua, &F.va, &F.delprsi, &F.delz, &F.wmp};
    const ShieldField3D* outs[] = {&F.pt_dt, &F.qv_dt, &F.ql_dt, &F.qr_dt, &F.qi_dt,
                                   &F.qs_dt, &F.qg_dt, &F.qa_dt, &F.udt,   &F.vdt};
    for (int f = 0; f < 13; ++f) {
      if (!ins[f]->ptr) {
        plan_free(p);
        return fail(nullptr, SHIELD_EINVAL, "member " + std::to_string(m) + ": null field");
      }
      A.in[f] = f3(*ins[f]);
    }
    for (int o = 0; o < 10; ++o) {
      if (!outs[o]->ptr) {
        plan_free(p);
        return fail(nullptr, SHIELD_EINVAL, "member " + std::to_string(m) + ": null tendency");
      }
      A.out[o] = f3(*outs[o]);
    }
    if (!F.land.ptr || A.K.de_ice) {
      plan_free(p);
      return fail(nullptr, SHIELD_EINVAL, "member " + std::to_string(m) + ": null land, or de_ice (not supported)");
    }
    A.out[OUT_W] = A.in[IN_W];
    A.land = Fld2{F.land.ptr, F.land.si, F.land.sj};
    A.rain = F.rain;
    A.snow = F.snow;
    A.ice = F.ice;
    A.graupel = F.graupel;
    area_off[m] = area_total;
    p->qaz_off[m] = qaz_total;
    area_total += A.ncol;
    qaz_total += A.ncol * nz;
  }
  p->qaz_total = qaz_total;
  if ((e = cudaMalloc(&p->d_area, sizeof(double) * area_total)) != cudaSuccess ||
      (e = cudaMalloc(&p->d_qaz, sizeof(double) * qaz_total)) != cudaSuccess ||
      (e = cudaMemset(p->d_qaz, 0, sizeof(double) * qaz_total)) != cudaSuccess ||
      (e = cudaMalloc(&p->d_members, sizeof(MpArgs) * nm)) != cudaSuccess ||
      (e = cudaMalloc(&p->d_counter, sizeof(unsigned long long))) != cudaSuccess) {
    int rc = cuda_fail(nullptr, e, "allocating the ensemble plan");
    plan_free(p);
    return rc;
  }
  for (int m = 0; m < nm; ++m) {
    MpArgs& A = host[m];
    A.area = Fld2{p->d_area + area_off[m], 1, A.nx};
    const Fld3 qaz{p->d_qaz + p->qaz_off[m], 1, A.nx, A.ncol};
    A.in[IN_QAZ] = qaz;
    A.out[OUT_QAZ] = qaz;
    e = mp_gather_area(mem[m].area.ptr, mem[m].area.si, mem[m].area.sj, A.nx, A.ny, p->d_area + area_off[m]);
    if (e != cudaSuccess) break;
  }
  if (e == cudaSuccess) e = cudaMemcpy(p->d_members, host.data(), sizeof(MpArgs) * nm, cudaMemcpyHostToDevice);
  const int Gs[5] = {1, 2, 4, 6, 8};
  for (int gi = 0; gi < 5 && e == cudaSuccess; ++gi) {
    std::vector<int64_t> offs(nm + 1, 0);
    for (int m = 0; m < nm; ++m) offs[m + 1] = offs[m] + (host[m].ncol + Gs[gi] - 1) / Gs[gi];
    e = cudaMalloc(&p->d_offs[gi], sizeof(int64_t) * (nm + 1));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->d_offs[gi], offs.data(), sizeof(int64_t) * (nm + 1), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    int rc = cuda_fail(nullptr, e, "uploading the ensemble plan");
    plan_free(p);
    return rc;
  }
  *plan = p;
  return SHIELD_OK;
}

extern "C" int shield_mp_ensemble_step(void* plan, int G, int bpsm, void* stream) {
  Plan* p = static_cast<Plan*>(plan);
  if (!p) return fail(nullptr, SHIELD_EINVAL, "null plan");
  const int gi = gindex(G);
  if (gi < 0 || !ensemble_shape_ok(p->nz, G) || bpsm < 1 || bpsm > 32)
    return fail(nullptr, SHIELD_EINVAL,
                std::string("cols_per_block must be ") + (p->nz <= 80 ? "2, 4, 6 or 8" : "1, 2 or 4") + " for " +
                    std::to_string(p->nz) + " levels, blocks_per_sm 1..32");
  const int grid = bpsm * p->num_sms;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = (p->precision == SHIELD_MP_MIXED)
                      ? mp_launch_ensemble_mixed(p->d_members, p->d_offs[gi], p->nm, p->nz, G, grid, p->d_counter, st)
                      : mp_launch_ensemble_plain(p->d_members, p->d_offs[gi], p->nm, p->nz, G, grid, p->d_counter, st);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "ensemble launch");
  return SHIELD_OK;
}

extern "C" int shield_mp_ensemble_qaz(void* plan, int m, double* out, void* stream) {
  Plan* p = static_cast<Plan*>(plan);
  if (!p || !out || m < 0 || m >= p->nm) return fail(nullptr, SHIELD_EINVAL, "bad arguments");
  const int64_t n = (m + 1 < p->nm ? p->qaz_off[m + 1] : p->qaz_total) - p->qaz_off[m];
  cudaError_t e = cudaMemcpyAsync(out, p->d_qaz + p->qaz_off[m], sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                  static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? SHIELD_OK : cuda_fail(nullptr, e, "copying qaz");
}

extern "C" int shield_mp_ensemble_destroy(void* plan) {
  Plan* p = static_cast<Plan*>(plan);
  if (p) plan_free(p);
  return SHIELD_OK;
}

// ------------------------------------------------------ allocation-free step
// shield_mp_step_noalloc: the step of shield_mp_step for callers that may not
// allocate device memory. Some hosts hand every byte of the GPU to their own
// pool or arena at start-up, and a cudaMalloc made behind its back either
// fails or breaks its accounting; others call physics from a context whose
// contract forbids allocation. The step's only scratch, the persistent
// cloud-fraction accumulator (nz values per column), therefore lives in the
// file-scope array below instead of a handle: it is part of this module's
// image, so the driver reserves it when the module loads on a GPU and every
// GPU that loads the library holds it until the process exits.
namespace {

// the largest nx * ny * nz the allocation-free step accepts: 16 MiB of
// accumulator (a 96 x 96 tile at 79 levels needs 0.73 M cells)
constexpr int64_t kNoAllocMaxCells = int64_t(1) << 21;
constexpr int kNoAllocMaxDevices = 64;

// accumulator cells, then one word for the kernel's error flag
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxCells + 32];

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// The array's device address on the current device. Its host-side name is
// only a stand-in, so the address is looked up with the device current. The
// first call on a device also clears the array; that clear runs on the
// legacy default stream and synchronises the device, so it is refused while
// the caller's stream is being captured. The lookup is repeated on every
// call (it allocates nothing): after a cudaDeviceReset the module is loaded
// again, possibly elsewhere, and a changed address repeats the set-up.
int noalloc_setup(int dev, cudaStream_t st, double** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  double* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetSymbolAddress of the allocation-free scratch");
  if (g_noalloc_ptr[dev] != p) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaStreamIsCapturing");
    if (cs != cudaStreamCaptureStatusNone)
      return fail(nullptr, SHIELD_EINVAL,
                  "the first allocation-free call on a device clears its scratch and synchronises the device; "
                  "make it before any stream capture");
    e = cudaMemset(p, 0, sizeof(g_noalloc_scratch));
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "clearing the allocation-free scratch");
    g_noalloc_ptr[dev] = p;
  }
  *out = p;
  return SHIELD_OK;
}

// The current device's scratch address and its validated ordinal, for the
// entry points below.
int noalloc_device(cudaStream_t st, double** scratch) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDevice");
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(nullptr, SHIELD_EINVAL, "device ordinal beyond 63");
  return noalloc_setup(dev, st, scratch);
}

}  // namespace

extern "C" int shield_mp_step_noalloc(const ShieldMpConfig* cfg, int nx, int ny, int nz, ShieldField2D area,
                                      const ShieldMpFields* F, double timestep, int precision, int first_step,
                                      void* stream) {
  if (!cfg || !F) return fail(nullptr, SHIELD_EINVAL, "null config or fields");
  if (nx < 1 || ny < 1) return fail(nullptr, SHIELD_EINVAL, "nx and ny must be positive");
  if (nz < 3 || nz > mp_max_levels()) return fail(nullptr, SHIELD_ELAYOUT, "nz must lie in [3, 256]");
  const int64_t ncol = (int64_t)nx * ny;
  if (ncol > kNoAllocMaxCells / nz)
    return fail(nullptr, SHIELD_ELAYOUT,
                "nx * ny * nz = " + std::to_string(ncol * nz) + " exceeds the allocation-free step's limit of " +
                    std::to_string(kNoAllocMaxCells) + " cells (its fixed 16 MiB scratch); use shield_mp_step");
  if (cfg->use_ppm) return fail(nullptr, SHIELD_EINVAL, "use_ppm=True is not supported (incomplete in the reference)");
  if (!area.ptr) return fail(nullptr, SHIELD_EINVAL, "null area pointer");
  if (precision != SHIELD_MP_PLAIN && precision != SHIELD_MP_MIXED)
    return fail(nullptr, SHIELD_EINVAL, "unknown precision mode");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* scratch = nullptr;
  int rc = noalloc_device(st, &scratch);
  if (rc != SHIELD_OK) return rc;
  cudaError_t e = cudaSuccess;

  MpArgs A;
  std::memset(&A, 0, sizeof(A));
  setupm(*cfg, A.K);
  std::string why;
  if (set_timestep(*cfg, A.K, timestep, why) != SHIELD_OK) return fail(nullptr, SHIELD_EINVAL, why);
  A.KF = to_float(A.K);
  A.nx = nx;
  A.ny = ny;
  A.nz = nz;
  A.ncol = ncol;
  const ShieldField3D* ins[] = {&F->pt, &F->qvapor, &F->qliquid, &F->qrain, &F->qice, &F->qsnow, &F->qgraupel,
                                &F->qcld, &F->ua, &F->va, &F->delprsi, &F->delz, &F->wmp};
  const ShieldField3D* outs[] = {&F->pt_dt, &F->qv_dt, &F->ql_dt, &F->qr_dt, &F->qi_dt,
                                 &F->qs_dt, &F->qg_dt, &F->qa_dt, &F->udt,   &F->vdt};
  for (int f = 0; f < 13; ++f) {
    if (!ins[f]->ptr) return fail(nullptr, SHIELD_EINVAL, "null input field pointer");
    A.in[f] = f3(*ins[f]);
  }
  for (int o = 0; o < 10; ++o) {
    if (!outs[o]->ptr) return fail(nullptr, SHIELD_EINVAL, "null tendency pointer");
    A.out[o] = f3(*outs[o]);
  }
  if (!F->land.ptr) return fail(nullptr, SHIELD_EINVAL, "null land pointer");
  // the accumulator, level-major over this call's nx * ny columns
  const Fld3 qaz{scratch, 1, nx, ncol};
  A.in[IN_QAZ] = qaz;
  A.out[OUT_W] = A.in[IN_W];
  A.out[OUT_QAZ] = qaz;
  A.land = Fld2{F->land.ptr, F->land.si, F->land.sj};
  A.area = Fld2{area.ptr, area.si, area.sj};
  A.rain = F->rain;
  A.snow = F->snow;
  A.ice = F->ice;
  A.graupel = F->graupel;
  A.err = reinterpret_cast<int*>(scratch + kNoAllocMaxCells);
  // The array keeps whatever the last call on this device left in it. The
  // first step of a run (or of another domain) starts from a zero
  // accumulator and a clear error word, as a freshly constructed handle does.
  if (first_step) {
    e = cudaMemsetAsync(scratch, 0, sizeof(double) * (size_t)(ncol * nz), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(A.err, 0, sizeof(int), st);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "clearing the accumulator");
  }
  if (A.K.de_ice) {
    e = mp_launch_de_ice(A, f3(F->qi_dt), f3(F->qs_dt), st);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "de_ice launch");
  }
  e = mp_launch_step(A, precision, st);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "microphysics launch");
  return SHIELD_OK;
}

// The allocation-free step's error word: the first column (+ 1) of any call
// since the last check (or since the last first_step call) that produced a
// NaN or an infinity. Read on `stream` after the calls queued on it.
extern "C" int shield_mp_check_noalloc(int nx, int64_t* bad_column, void* stream) {
  if (bad_column) *bad_column = -1;
  if (nx < 1) return fail(nullptr, SHIELD_EINVAL, "nx must be positive");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* scratch = nullptr;
  int rc = noalloc_device(st, &scratch);
  if (rc != SHIELD_OK) return rc;
  int* err = reinterpret_cast<int*>(scratch + kNoAllocMaxCells);
  int v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "reading the allocation-free error word");
  if (v == 0) return SHIELD_OK;
  e = cudaMemsetAsync(err, 0, sizeof(int), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "clearing the allocation-free error word");
  const int64_t c = (int64_t)v - 1;
  if (bad_column) *bad_column = c;
  return fail(nullptr, SHIELD_EDEVICE,
              "column " + std::to_string(c) + " (i = " + std::to_string(c % nx) + ", j = " + std::to_string(c / nx) +
                  ") produced a NaN or an infinity");
}
