// fr_solver.cu -- the fr_solver object behind the C ABI of include/fr_b200.h:
// device buffers, template dispatch over (dims, order, precision), the RK45
// driver with CUDA-graph replay, reductions.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "fr_b200.h"
#include "fr_runner.cuh"

namespace frb {

thread_local std::string g_err;

// blocks of the integral-diagnostics kernel (partial sums added in block order)
constexpr int kDiagBlocks = 296;

cudaError_t launch_sgs_inputs(int dims, int tc_size, const double* U, const void* G, const double* detj, long long npts,
                              int nu, long long E, int order, double filter_ratio, float* X, cudaStream_t st);
void mlp_default_params(float* w);
cudaError_t launch_diagnostics(int dims, int tc_size, const double* U, const void* G, const double* opp,
                               const double* W, const double* detj, long long E, int nu, int nc, double gamma,
                               double* partial, int nblk, double* out, cudaStream_t st);

static fr_status fail(fr_status s, const std::string& msg)
{
  g_err = msg;
  return s;
}

#define FR_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return fail(FR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)

static Runner* make_runner(int dims, int P, int tc_size, long long E, int visc, int les, const Line1D& l,
                           const Phys& p)
{
#define FR_CASE(D_, P_, T_) \
  if (dims == D_ && P == P_ && tc_size == (int)sizeof(T_)) return FR_RUNNER_NAME(D_, P_, T_)(E, visc, les, l, p);
  FR_CASE(2, 1, double) FR_CASE(2, 2, double) FR_CASE(2, 3, double) FR_CASE(2, 4, double) FR_CASE(2, 5, double)
  FR_CASE(3, 1, double) FR_CASE(3, 2, double) FR_CASE(3, 3, double) FR_CASE(3, 4, double)
  FR_CASE(2, 1, float) FR_CASE(2, 2, float) FR_CASE(2, 3, float) FR_CASE(2, 4, float) FR_CASE(2, 5, float)
  FR_CASE(3, 1, float) FR_CASE(3, 2, float) FR_CASE(3, 3, float) FR_CASE(3, 4, float)
#undef FR_CASE
  return nullptr;
}

}  // namespace frb

using namespace frb;

struct fr_solver {
  int device = 0;
  fr_scheme_desc sch{};
  Line1D line;
  Mesh mesh;
  Bufs b;
  std::unique_ptr<Runner> run;
  size_t tc_size = 8;
  int cur = 0;                      // trace buffer holding the current state's traces
  cudaStream_t own_stream = nullptr; // used when the caller passes stream == NULL
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  double graph_dt[2] = {0, 0};
  long long launches = 0;
  // volume cubature of the integral diagnostics (reference volume_cub_order
  // 3 by default): points (dims, nc), weights, and on the device the
  // interpolation rows, weights and Jacobians at the cubature points
  int vc_n = 0;
  std::vector<double> vc_loc, vc_w;
  bool vc_dirty = true;
  double *vc_opp = nullptr, *vc_wd = nullptr, *vc_detj = nullptr;
  float* mlp = nullptr;             // learned-closure parameters (sgs_model 5)
  void* grad_buf = nullptr;         // gradient output of fr_solver_gradient (allocated on first use)
  float* feat_buf = nullptr;        // closure inputs of fr_solver_sgs_features (allocated on first use)
  double *diag_partial = nullptr, *diag_out = nullptr;   // integral diagnostics
  // asynchronous state upload (fr_solver_set_state_async): a device staging
  // copy of the state, filled on its own stream while earlier steps run
  double* staging = nullptr;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_staged = nullptr, ev_consumed = nullptr;
  bool staged = false;
  std::vector<void*> allocs;
};

#define STRM(s, stream) ((stream) ? (cudaStream_t)(stream) : (s)->own_stream)

namespace {

template <typename T>
fr_status dalloc(fr_solver* s, T** p, size_t n)
{
  void* q = nullptr;
  FR_CUDA(cudaMalloc(&q, n * sizeof(T) + 16));
  s->allocs.push_back(q);
  *p = (T*)q;
  return FR_OK;
}

fr_status upload_tc(fr_solver* s, void* dst, const std::vector<double>& src)
{
  if (s->tc_size == 8) {
    FR_CUDA(cudaMemcpy(dst, src.data(), src.size() * 8, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> f(src.begin(), src.end());
    FR_CUDA(cudaMemcpy(dst, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
  }
  return FR_OK;
}

fr_status upload_geometry(fr_solver* s)
{
  Mesh& m = s->mesh;
  fr_status st;
  if ((st = upload_tc(s, s->b.JG, m.JG))) return st;
  if ((st = upload_tc(s, s->b.detj, m.detjac))) return st;
  if ((st = upload_tc(s, s->b.tdA, m.tdA))) return st;
  if ((st = upload_tc(s, s->b.nL, m.nL))) return st;
  FR_CUDA(cudaMemcpy(s->b.detj64, m.detjac.data(), m.detjac.size() * 8, cudaMemcpyHostToDevice));
  {
    std::vector<double> inv(m.detjac.size());
    for (size_t i = 0; i < inv.size(); i++) inv[i] = 1.0 / m.detjac[i];
    FR_CUDA(cudaMemcpy(s->b.idetj, inv.data(), inv.size() * 8, cudaMemcpyHostToDevice));
  }
  FR_CUDA(cudaMemcpy(s->b.mate, m.mate.data(), m.mate.size() * sizeof(int), cudaMemcpyHostToDevice));
  std::vector<unsigned char> side(m.mate.size());
  size_t E = m.ne;
  for (size_t i = 0; i < side.size(); i++) {
    size_t f = i % m.nf, e = i / m.nf;
    double n[3] = {0, 0, 0};
    for (int d = 0; d < m.dims; d++) n[d] = m.nL[f + m.nf * (e + E * d)];
    // sign switch of the LDG penalty from the left normal (src/inters.cpp:555-564)
    double sgn = m.dims == 2 ? (n[0] + n[1]) : (n[0] + n[1] + std::sqrt(2.) * n[2]);
    side[i] = (m.is_left[i] ? 1 : 0) | (sgn < 0. ? 2 : 0);
  }
  for (size_t j = 0; j < m.bf.size(); j++) side[m.bf[j]] = (unsigned char)(1 | (m.bt[j] << 2));
  FR_CUDA(cudaMemcpy(s->b.side, side.data(), side.size(), cudaMemcpyHostToDevice));
  std::vector<int2> face(m.il.size());
  std::vector<unsigned char> fsign(m.il.size());
  for (size_t i = 0; i < face.size(); i++) {
    face[i] = make_int2(m.il[i], m.ir[i]);
    fsign[i] = (side[m.il[i]] & 2) ? 1 : 0;
  }
  FR_CUDA(cudaMemcpy(s->b.face, face.data(), face.size() * sizeof(int2), cudaMemcpyHostToDevice));
  FR_CUDA(cudaMemcpy(s->b.fsign, fsign.data(), fsign.size(), cudaMemcpyHostToDevice));
  if (s->b.nbdy > 0) {
    FR_CUDA(cudaMemcpy(s->b.bf, m.bf.data(), m.bf.size() * sizeof(int), cudaMemcpyHostToDevice));
    FR_CUDA(cudaMemcpy(s->b.bt, m.bt.data(), m.bt.size(), cudaMemcpyHostToDevice));
  }
  return FR_OK;
}

void drop_graphs(fr_solver* s)
{
  for (int i = 0; i < 2; i++)
    if (s->graph[i]) { cudaGraphExecDestroy(s->graph[i]); s->graph[i] = nullptr; }
}

fr_status check_launch(const char* what)
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(FR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FR_OK;
}

// A kernel whose bounded wait gave up has set the solver's error flag; read
// (and clear) it at the points where the host waits for the device anyway.
fr_status check_device_flag(fr_solver* s, cudaStream_t st)
{
  int h = 0;
  FR_CUDA(cudaMemcpyAsync(&h, s->b.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  FR_CUDA(cudaStreamSynchronize(st));
  if (h) {
    FR_CUDA(cudaMemsetAsync(s->b.err, 0, sizeof(int), st));
    return fail(FR_ERR_TIMEOUT, "a stage kernel's wait for its bulk copies timed out");
  }
  return FR_OK;
}

// one RK stage: residual + update; traces flip buffers
fr_status stage(fr_solver* s, int st, double dt, bool want_partial, cudaStream_t stream)
{
  if (s->sch.viscous) { s->run->grad(s->b, s->cur, stream); s->launches++; }
  s->run->face(s->b, s->cur, stream);
  s->run->update(s->b, s->cur, 1, st, dt, want_partial, stream);
  s->launches += 2;
  s->cur ^= 1;
  return check_launch("fr stage kernels");
}

}  // namespace

static fr_status create_with_mesh(Mesh&& mesh, const Line1D& line, const fr_scheme_desc* sd, int device,
                                  fr_solver** out);
static fr_status validate_scheme(int dims, const fr_scheme_desc* sd);

extern "C" {

const char* fr_status_string(fr_status s)
{
  switch (s) {
    case FR_OK: return "ok";
    case FR_ERR_ARG: return "invalid argument";
    case FR_ERR_CUDA: return "CUDA error";
    case FR_ERR_NONFINITE: return "non-finite residual";
    case FR_ERR_TIMEOUT: return "device wait timed out";
    case FR_ERR_UNSUPPORTED: return "unsupported configuration";
    case FR_ERR_MESH: return "mesh wiring failed";
  }
  return "unknown status";
}

const char* fr_last_error(void) { return g_err.c_str(); }

fr_status fr_solver_create(const fr_mesh_desc* md, const fr_scheme_desc* sd, int device, fr_solver** out)
{
  g_err.clear();
  if (!md || !sd || !out) return fail(FR_ERR_ARG, "null argument");
  *out = nullptr;
  fr_status v = validate_scheme(md->dims, sd);
  if (v) return v;
  Line1D line;
  std::string err;
  if (!make_line(sd->order, sd->upts_type, sd->vcjh_scheme, sd->eta, line, err)) return fail(FR_ERR_ARG, err);
  Mesh mesh;
  if (!build_mesh(md->dims, line, md->n_verts, md->xv, md->n_eles, md->c2v, md->shift, md->bctype, mesh, err))
    return fail(FR_ERR_MESH, err);
  return create_with_mesh(std::move(mesh), line, sd, device, out);
}

}  // extern "C"

static fr_status validate_scheme(int dims, const fr_scheme_desc* sd)
{
  if (dims != 2 && dims != 3) return fail(FR_ERR_ARG, "dims must be 2 or 3");
  if (sd->riemann != 0 && !(sd->riemann == 2 && dims == 2))
    return fail(FR_ERR_UNSUPPORTED, "common fluxes built: Rusanov (0), and Roe (2) in 2-D as in the reference");
  if (sd->precision != 0 && sd->precision != 1) return fail(FR_ERR_ARG, "precision must be 0 or 1");
  int maxP = dims == 2 ? 5 : 4;
  if (sd->order < 1 || sd->order > maxP) return fail(FR_ERR_UNSUPPORTED, "order outside the built range");
  if (sd->upts_type != 0) return fail(FR_ERR_UNSUPPORTED, "fused kernels need Gauss solution points");
  if (sd->les != 0) {
    if (sd->les != 1 || !sd->viscous) return fail(FR_ERR_ARG, "les must be 0 or 1, and 1 needs viscous = 1");
    if (sd->sgs_model != 0 && sd->sgs_model != 1 && sd->sgs_model != 5)
      return fail(FR_ERR_UNSUPPORTED,
                  "SGS models built: 0 (Smagorinsky), 1 (WALE) and 5 (learned); the filter-based models are not");
    if (!(sd->filter_ratio > 0.0)) return fail(FR_ERR_ARG, "filter_ratio must be positive");
  }
  return FR_OK;
}

// Everything of fr_solver_create after the mesh is wired (also used for the
// merged meshes of a batch).
static fr_status create_with_mesh(Mesh&& mesh, const Line1D& line, const fr_scheme_desc* sd, int device,
                                  fr_solver** out)
{
  std::unique_ptr<fr_solver> s(new fr_solver());
  s->device = device;
  s->sch = *sd;
  s->tc_size = sd->precision == 1 ? 4 : 8;
  s->line = line;
  s->mesh = std::move(mesh);
  FR_CUDA(cudaSetDevice(device));
  if (sd->les && sd->sgs_model == 5) {
    // the learned closure starts switched off (c ~ 2e-9) until parameters are set
    fr_status st0 = dalloc(s.get(), &s->mlp, (size_t)kMlpN);
    if (st0) return st0;
    std::vector<float> w0(kMlpN);
    mlp_default_params(w0.data());
    FR_CUDA(cudaMemcpy(s->mlp, w0.data(), sizeof(float) * kMlpN, cudaMemcpyHostToDevice));
  }
  Phys ph{sd->gamma, sd->prandtl, sd->mu_inf, sd->rt_inf, sd->c_sth, sd->fix_vis, sd->tau, sd->pen_fact,
          sd->sgs_model, sd->filter_ratio, s->mlp};
  for (int i = 0; i < 14; i++) ph.bdy[i] = sd->bdy[i];
  ph.R_ref = sd->R_ref;
  const int les = sd->les;
  Runner* r = make_runner(s->mesh.dims, sd->order, (int)s->tc_size, s->mesh.ne, sd->viscous, les, s->line, ph);
  if (!r) return fail(FR_ERR_UNSUPPORTED, "no kernel for this (dims, order)");
  r->set_riemann(sd->riemann);
  s->run.reset(r);
  Mesh& m = s->mesh;
  size_t E = m.ne, F = m.nfields, D = m.dims, nu = m.nu, nf = m.nf, tc = s->tc_size;
  fr_status st;
  if ((st = dalloc(s.get(), &s->b.U, nu * E * F))) return st;
  if ((st = dalloc(s.get(), &s->b.REG, nu * E * F))) return st;
  if ((st = dalloc(s.get(), &s->b.DIV, nu * E * F))) return st;
  if ((st = dalloc(s.get(), &s->b.detj64, nu * E))) return st;
  if ((st = dalloc(s.get(), &s->b.idetj, nu * E))) return st;
  if ((st = dalloc(s.get(), &s->b.err, 1))) return st;
  char* p;
  for (int i = 0; i < 2; i++) { if ((st = dalloc(s.get(), &p, nf * E * F * tc))) return st; s->b.UF[i] = p; }
  if (sd->viscous) {
    if ((st = dalloc(s.get(), &p, nf * E * (F - 1) * tc))) return st; s->b.VF = p;
    if ((st = dalloc(s.get(), &p, nf * E * F * tc))) return st; s->b.ND = p;
    if ((st = dalloc(s.get(), &p, nu * E * F * tc))) return st; s->b.DV = p;
  }
  if ((st = dalloc(s.get(), &p, nf * E * F * tc))) return st; s->b.CF = p;
  s->b.nint = (long long)m.il.size();
  s->b.nbdy = (long long)m.bf.size();
  if (s->b.nbdy > 0) {
    if ((st = dalloc(s.get(), &s->b.bf, (size_t)s->b.nbdy))) return st;
    if ((st = dalloc(s.get(), &s->b.bt, (size_t)s->b.nbdy))) return st;
    if (sd->viscous) { if ((st = dalloc(s.get(), &p, (size_t)s->b.nbdy * F * tc))) return st; s->b.BV = p; }
  }
  if ((st = dalloc(s.get(), &s->b.face, (size_t)s->b.nint))) return st;
  if ((st = dalloc(s.get(), &s->b.fsign, (size_t)s->b.nint))) return st;
  if ((st = dalloc(s.get(), &p, nf * E * D * tc))) return st; s->b.nL = p;
  if ((st = dalloc(s.get(), &p, nf * E * tc))) return st; s->b.tdA = p;
  if ((st = dalloc(s.get(), &p, D * D * nu * E * tc))) return st; s->b.JG = p;
  if ((st = dalloc(s.get(), &p, nu * E * tc))) return st; s->b.detj = p;
  if ((st = dalloc(s.get(), &s->b.mate, nf * E))) return st;
  if ((st = dalloc(s.get(), &s->b.side, nf * E))) return st;
  if ((st = dalloc(s.get(), &s->b.partial, (size_t)s->run->max_flux_blocks() * F))) return st;
  if ((st = dalloc(s.get(), &s->b.norms, F))) return st;
  s->vc_n = volume_cubature(m.dims, 3, s->vc_loc, s->vc_w);
  if ((st = dalloc(s.get(), &s->diag_partial, (size_t)kDiagBlocks * 5))) return st;
  if ((st = dalloc(s.get(), &s->diag_out, 5))) return st;
  FR_CUDA(cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking));
  FR_CUDA(cudaMemset(s->b.err, 0, sizeof(int)));
  FR_CUDA(cudaMemset(s->b.U, 0, nu * E * F * 8));
  FR_CUDA(cudaMemset(s->b.REG, 0, nu * E * F * 8));
  if ((st = upload_geometry(s.get()))) return st;
  *out = s.release();
  return FR_OK;
}

extern "C" {

fr_status fr_solver_destroy(fr_solver* s)
{
  if (!s) return FR_OK;
  cudaSetDevice(s->device);
  drop_graphs(s);
  if (s->own_stream) { cudaStreamSynchronize(s->own_stream); cudaStreamDestroy(s->own_stream); }
  if (s->copy_stream) { cudaStreamSynchronize(s->copy_stream); cudaStreamDestroy(s->copy_stream); }
  if (s->ev_staged) cudaEventDestroy(s->ev_staged);
  if (s->ev_consumed) cudaEventDestroy(s->ev_consumed);
  for (void* p : s->allocs) cudaFree(p);
  delete s;
  return FR_OK;
}

fr_status fr_solver_sizes(const fr_solver* s, int out[6])
{
  if (!s || !out) return fail(FR_ERR_ARG, "null argument");
  out[0] = (int)s->mesh.ne; out[1] = s->mesh.nu; out[2] = s->mesh.nf; out[3] = s->mesh.nfields;
  out[4] = s->mesh.dims; out[5] = (int)s->mesh.il.size();
  return FR_OK;
}

fr_status fr_solver_get_geometry(const fr_solver* s, double* pos, double* detj, double* JG, double* tdA, double* nrm)
{
  if (!s) return fail(FR_ERR_ARG, "null solver");
  const Mesh& m = s->mesh;
  if (pos) memcpy(pos, m.pos_upts.data(), m.pos_upts.size() * 8);
  if (detj) memcpy(detj, m.detjac.data(), m.detjac.size() * 8);
  if (JG) memcpy(JG, m.JG.data(), m.JG.size() * 8);
  if (tdA) memcpy(tdA, m.tdA.data(), m.tdA.size() * 8);
  if (nrm) memcpy(nrm, m.nrm.data(), m.nrm.size() * 8);
  return FR_OK;
}

fr_status fr_solver_get_interfaces(const fr_solver* s, int* l, int* r)
{
  if (!s || !l || !r) return fail(FR_ERR_ARG, "null argument");
  memcpy(l, s->mesh.il.data(), s->mesh.il.size() * sizeof(int));
  memcpy(r, s->mesh.ir.data(), s->mesh.ir.size() * sizeof(int));
  return FR_OK;
}

fr_status fr_solver_set_geometry(fr_solver* s, const double* detj, const double* JG, const double* tdA,
                                 const double* nrm)
{
  if (!s || !detj || !JG || !tdA || !nrm) return fail(FR_ERR_ARG, "null argument");
  Mesh& m = s->mesh;
  for (size_t i = 0; i < m.detjac.size(); i++)
    if (!(detj[i] > 0)) return fail(FR_ERR_ARG, "non-positive Jacobian");
  memcpy(m.detjac.data(), detj, m.detjac.size() * 8);
  memcpy(m.JG.data(), JG, m.JG.size() * 8);
  memcpy(m.tdA.data(), tdA, m.tdA.size() * 8);
  memcpy(m.nrm.data(), nrm, m.nrm.size() * 8);
  finish_wiring(m);
  FR_CUDA(cudaSetDevice(s->device));
  drop_graphs(s);
  s->vc_dirty = true;
  return upload_geometry(s);
}

fr_status fr_solver_state_ptrs(fr_solver* s, double** u, double** reg)
{
  if (!s) return fail(FR_ERR_ARG, "null solver");
  if (u) *u = s->b.U;
  if (reg) *reg = s->b.REG;
  return FR_OK;
}

fr_status fr_solver_state_updated(fr_solver* s, void* stream)
{
  if (!s) return fail(FR_ERR_ARG, "null solver");
  FR_CUDA(cudaSetDevice(s->device));
  s->run->trace(s->b, s->cur, STRM(s, stream));
  s->launches++;
  return check_launch("fr_trace_kernel");
}

// Every density positive and finite; large arrays are split over host threads.
static bool densities_ok(const double* rho, size_t n)
{
  auto scan = [rho](size_t a, size_t b) {
    bool ok = true;
    for (size_t i = a; i < b; i++) ok &= (rho[i] > 0) && std::isfinite(rho[i]);
    return ok;
  };
  unsigned nt = std::thread::hardware_concurrency();
  nt = nt < 1 ? 1 : (nt > 16 ? 16 : nt);
  if (n < (size_t)1 << 18 || nt == 1) return scan(0, n);
  std::vector<std::thread> pool;
  std::vector<char> ok(nt, 1);
  const size_t chunk = (n + nt - 1) / nt;
  for (unsigned t = 0; t < nt; t++) {
    const size_t a = t * chunk, b = a + chunk < n ? a + chunk : n;
    pool.emplace_back([&, t, a, b] { ok[t] = a < b ? scan(a, b) : 1; });
  }
  for (auto& th : pool) th.join();
  for (char c : ok)
    if (!c) return false;
  return true;
}

fr_status fr_solver_set_state(fr_solver* s, const double* host_u, void* stream)
{
  if (!s || !host_u) return fail(FR_ERR_ARG, "null argument");
  FR_CUDA(cudaSetDevice(s->device));
  size_t n = (size_t)s->mesh.nu * s->mesh.ne * s->mesh.nfields;
  if (!densities_ok(host_u, (size_t)s->mesh.nu * s->mesh.ne))
    return fail(FR_ERR_NONFINITE, "density must be positive and finite");
  cudaStream_t st = STRM(s, stream);
  FR_CUDA(cudaMemcpyAsync(s->b.U, host_u, n * 8, cudaMemcpyHostToDevice, st));
  FR_CUDA(cudaMemsetAsync(s->b.REG, 0, n * 8, st));
  return fr_solver_state_updated(s, stream);
}

fr_status fr_solver_set_state_async(fr_solver* s, const double* host_u)
{
  if (!s || !host_u) return fail(FR_ERR_ARG, "null argument");
  FR_CUDA(cudaSetDevice(s->device));
  size_t n = (size_t)s->mesh.nu * s->mesh.ne * s->mesh.nfields;
  if (!densities_ok(host_u, (size_t)s->mesh.nu * s->mesh.ne))
    return fail(FR_ERR_NONFINITE, "density must be positive and finite");
  if (!s->staging) {
    fr_status r = dalloc(s, &s->staging, n);
    if (r) return r;
    FR_CUDA(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
    FR_CUDA(cudaEventCreateWithFlags(&s->ev_staged, cudaEventDisableTiming));
    FR_CUDA(cudaEventCreateWithFlags(&s->ev_consumed, cudaEventDisableTiming));
    FR_CUDA(cudaEventRecord(s->ev_consumed, s->copy_stream));
  }
  if (s->staged) return fail(FR_ERR_ARG, "a staged state has not been taken by an advance yet");
  // the staging buffer is free once the step that took the previous state has copied it
  FR_CUDA(cudaStreamWaitEvent(s->copy_stream, s->ev_consumed, 0));
  FR_CUDA(cudaMemcpyAsync(s->staging, host_u, n * 8, cudaMemcpyHostToDevice, s->copy_stream));
  FR_CUDA(cudaEventRecord(s->ev_staged, s->copy_stream));
  s->staged = true;
  return FR_OK;
}

// The staged state (if any) becomes the current state, in stream order: one
// pass copies it into place and extrapolates its traces.  The RK register
// is left as it is: the first stage of a step writes it without reading it.
static fr_status take_staged(fr_solver* s, cudaStream_t st)
{
  if (!s->staged) return FR_OK;
  FR_CUDA(cudaStreamWaitEvent(st, s->ev_staged, 0));
  s->run->trace(s->b, s->cur, st, s->staging);
  s->launches++;
  if (fr_status r = check_launch("fr_trace_kernel")) return r;
  FR_CUDA(cudaEventRecord(s->ev_consumed, st));
  s->staged = false;
  return FR_OK;
}

fr_status fr_solver_get_state(fr_solver* s, double* host_u, void* stream)
{
  if (!s || !host_u) return fail(FR_ERR_ARG, "null argument");
  FR_CUDA(cudaSetDevice(s->device));
  size_t n = (size_t)s->mesh.nu * s->mesh.ne * s->mesh.nfields;
  FR_CUDA(cudaMemcpyAsync(host_u, s->b.U, n * 8, cudaMemcpyDeviceToHost, STRM(s, stream)));
  FR_CUDA(cudaStreamSynchronize(STRM(s, stream)));
  return FR_OK;
}

fr_status fr_solver_residual(fr_solver* s, double* host_div, void* stream)
{
  if (!s || !host_div) return fail(FR_ERR_ARG, "null argument");
  FR_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = STRM(s, stream);
  if (s->sch.viscous) { s->run->grad(s->b, s->cur, st); s->launches++; }
  s->run->face(s->b, s->cur, st);
  s->run->update(s->b, s->cur, 0, 0, 0.0, false, st);
  s->launches += 2;
  fr_status r = check_launch("fr residual kernels");
  if (r) return r;
  size_t n = (size_t)s->mesh.nu * s->mesh.ne * s->mesh.nfields;
  FR_CUDA(cudaMemcpyAsync(host_div, s->b.DIV, n * 8, cudaMemcpyDeviceToHost, st));
  FR_CUDA(cudaStreamSynchronize(st));
  return check_device_flag(s, st);
}

fr_status fr_solver_rk_stage(fr_solver* s, int st, double dt, void* stream)
{
  if (!s || st < 0 || st > 4) return fail(FR_ERR_ARG, "stage must be 0..4");
  FR_CUDA(cudaSetDevice(s->device));
  return stage(s, st, dt, st == 4, STRM(s, stream));
}

static fr_status advance_impl(fr_solver* s, int n_steps, double dt, double* norms_host, void* stream, bool wait);

fr_status fr_solver_advance(fr_solver* s, int n_steps, double dt, double* norms_host, void* stream)
{
  return advance_impl(s, n_steps, dt, norms_host, stream, true);
}

fr_status fr_solver_advance_async(fr_solver* s, int n_steps, double dt, double* norms_host, void* stream)
{
  return advance_impl(s, n_steps, dt, norms_host, stream, false);
}

static fr_status advance_impl(fr_solver* s, int n_steps, double dt, double* norms_host, void* stream, bool wait)
{
  if (!s || n_steps < 0) return fail(FR_ERR_ARG, "bad argument");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(FR_ERR_ARG, "dt must be positive");
  FR_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = STRM(s, stream);
  {
    fr_status r = take_staged(s, st);
    if (r) return r;
  }
  bool capture_ok = true;
  for (int i = 0; i < n_steps; i++) {
    int c = s->cur;
    if (capture_ok && (!s->graph[c] || s->graph_dt[c] != dt)) {
      if (s->graph[c]) { cudaGraphExecDestroy(s->graph[c]); s->graph[c] = nullptr; }
      cudaGraph_t g;
      FR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      long long l0 = s->launches;
      for (int k = 0; k < 5; k++) stage(s, k, dt, k == 4, st);
      s->launches = l0;
      s->cur = c;
      FR_CUDA(cudaStreamEndCapture(st, &g));
      cudaError_t e = cudaGraphInstantiate(&s->graph[c], g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return fail(FR_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      s->graph_dt[c] = dt;
    }
    if (capture_ok) {
      FR_CUDA(cudaGraphLaunch(s->graph[c], st));
      s->launches += 5 * s->run->launches_per_stage();
      s->cur ^= 1;   // five stages: an odd number of trace-buffer flips
    } else {
      for (int k = 0; k < 5; k++) {
        fr_status r = stage(s, k, dt, k == 4, st);
        if (r) return r;
      }
    }
  }
  if (norms_host) {
    int F = s->mesh.nfields;
    double inv_n = 1.0 / ((double)s->mesh.nu * (double)s->mesh.ne);
    fr_norm_finalize<<<F, 256, 0, st>>>(s->b.partial, s->run->flux_blocks(), F, inv_n, s->b.norms);
    s->launches++;
    FR_CUDA(cudaGetLastError());
    FR_CUDA(cudaMemcpyAsync(norms_host, s->b.norms, F * 8, cudaMemcpyDeviceToHost, st));
    if (!wait) return FR_OK;
    FR_CUDA(cudaStreamSynchronize(st));
    fr_status fl = check_device_flag(s, st);
    if (fl) return fl;
    for (int k = 0; k < F; k++)
      if (!std::isfinite(norms_host[k])) return fail(FR_ERR_NONFINITE, "NaN/Inf in the residual");
  }
  return FR_OK;
}

// The device copies of the volume cubature (interpolation rows, weights,
// Jacobians at the cubature points), rebuilt after the rule or the geometry changed.
static fr_status volume_cubature_ready(fr_solver* s)
{
  if (!s->vc_dirty) return FR_OK;
  const Mesh& m = s->mesh;
  std::vector<double> opp, dj;
  volume_cubature_setup(m, s->line, s->vc_n, s->vc_loc.data(), opp, dj);
  for (void* p : {(void*)s->vc_opp, (void*)s->vc_wd, (void*)s->vc_detj})
    if (p) {
      for (size_t i = 0; i < s->allocs.size(); i++)
        if (s->allocs[i] == p) { s->allocs.erase(s->allocs.begin() + i); break; }
      cudaFree(p);
    }
  s->vc_opp = s->vc_wd = s->vc_detj = nullptr;
  fr_status r;
  if ((r = dalloc(s, &s->vc_opp, opp.size()))) return r;
  if ((r = dalloc(s, &s->vc_wd, s->vc_w.size()))) return r;
  if ((r = dalloc(s, &s->vc_detj, dj.size()))) return r;
  FR_CUDA(cudaMemcpy(s->vc_opp, opp.data(), opp.size() * 8, cudaMemcpyHostToDevice));
  FR_CUDA(cudaMemcpy(s->vc_wd, s->vc_w.data(), s->vc_w.size() * 8, cudaMemcpyHostToDevice));
  FR_CUDA(cudaMemcpy(s->vc_detj, dj.data(), dj.size() * 8, cudaMemcpyHostToDevice));
  s->vc_dirty = false;
  return FR_OK;
}

fr_status fr_solver_kinetic_energy(fr_solver* s, double* out, void* stream)
{
  if (!s || !out) return fail(FR_ERR_ARG, "null argument");
  FR_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = STRM(s, stream);
  fr_status r = volume_cubature_ready(s);
  if (r) return r;
  const Mesh& m = s->mesh;
  FR_CUDA(launch_diagnostics(m.dims, (int)s->tc_size, s->b.U, nullptr, s->vc_opp, s->vc_wd, s->vc_detj, m.ne, m.nu,
                             s->vc_n, s->sch.gamma, s->diag_partial, kDiagBlocks, s->diag_out, st));
  s->launches += 2;
  FR_CUDA(cudaMemcpyAsync(out, s->diag_out, 8, cudaMemcpyDeviceToHost, st));
  FR_CUDA(cudaStreamSynchronize(st));
  return FR_OK;
}

fr_status fr_solver_set_volume_cubature(fr_solver* s, int n_cub, const double* loc, const double* weights)
{
  if (!s || n_cub <= 0 || !loc || !weights) return fail(FR_ERR_ARG, "bad argument");
  const int D = s->mesh.dims;
  for (int i = 0; i < n_cub * D; i++)
    if (!(loc[i] >= -1.0 && loc[i] <= 1.0)) return fail(FR_ERR_ARG, "cubature points must lie in [-1, 1]");
  s->vc_n = n_cub;
  s->vc_loc.assign(loc, loc + (size_t)n_cub * D);
  s->vc_w.assign(weights, weights + n_cub);
  s->vc_dirty = true;
  return FR_OK;
}

int fr_volume_cubature(int dims, int rule, double* loc, double* weights)
{
  std::vector<double> l, w;
  const int n = volume_cubature(dims, rule, l, w);
  if (n > 0) {
    if (loc) memcpy(loc, l.data(), l.size() * 8);
    if (weights) memcpy(weights, w.data(), w.size() * 8);
  }
  return n;
}

long long fr_solver_launch_count(const fr_solver* s) { return s ? s->launches : 0; }

void* fr_solver_stream(fr_solver* s) { return s ? (void*)s->own_stream : nullptr; }

fr_status fr_solver_profile_stage(fr_solver* s, int reps, double dt, double* ms3)
{
  if (!s || reps <= 0 || !ms3) return fail(FR_ERR_ARG, "bad argument");
  FR_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = s->own_stream;
  cudaEvent_t ev[4];
  for (int i = 0; i < 4; i++) FR_CUDA(cudaEventCreate(&ev[i]));
  double acc[3] = {0, 0, 0};
  for (int r = 0; r < reps; r++) {
    int k = r % 5;
    FR_CUDA(cudaEventRecord(ev[0], st));
    if (s->sch.viscous) { s->run->grad(s->b, s->cur, st); s->launches++; }
    FR_CUDA(cudaEventRecord(ev[1], st));
    s->run->face(s->b, s->cur, st);
    FR_CUDA(cudaEventRecord(ev[2], st));
    s->run->update(s->b, s->cur, 1, k, dt, k == 4, st);
    s->launches += 2;
    s->cur ^= 1;
    FR_CUDA(cudaEventRecord(ev[3], st));
    FR_CUDA(cudaEventSynchronize(ev[3]));
    for (int i = 0; i < 3; i++) {
      float ms = 0.f;
      FR_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
      acc[i] += ms;
    }
  }
  for (int i = 0; i < 4; i++) cudaEventDestroy(ev[i]);
  FR_CUDA(cudaGetLastError());
  for (int i = 0; i < 3; i++) ms3[i] = acc[i] / reps;
  return FR_OK;
}

fr_status fr_solver_autotune(fr_solver* s, int reps, int out4[4])
{
  if (!s || reps <= 0) return fail(FR_ERR_ARG, "bad argument");
  FR_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = s->own_stream;
  cudaEvent_t a, b;
  FR_CUDA(cudaEventCreate(&a));
  FR_CUDA(cudaEventCreate(&b));
  auto time_it = [&](auto&& launch) -> double {
    launch();                                  // warm-up (and shared-memory opt-in)
    cudaEventRecord(a, st);
    for (int r = 0; r < reps; r++) launch();
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms / reps;
  };
  Runner* R = s->run.get();
  int g0 = R->grad_sel(), u0 = R->update_sel();
  // the gradient kernel only writes scratch (VF, ND, DV) and the update kernel
  // in residual mode only writes DIV, so timing them leaves the state as it is
  int gbest = g0;
  if (s->sch.viscous) {
    double best = 1e30;
    for (int g = 0; g < R->n_grad_tiles(); g++) {
      R->select(g, u0);
      double ms = time_it([&] { R->grad(s->b, s->cur, st); s->launches++; });
      if (ms < best) { best = ms; gbest = g; }
    }
    R->select(gbest, u0);
    R->grad(s->b, s->cur, st);                 // scratch consistent with the current state
    s->launches++;
  }
  int ubest = u0;
  {
    double best = 1e30;
    for (int u = 0; u < R->n_update_tiles(); u++) {
      R->select(gbest, u);
      double ms = time_it([&] { R->update(s->b, s->cur, 0, 0, 0.0, false, st); s->launches++; });
      if (ms < best) { best = ms; ubest = u; }
    }
  }
  R->select(gbest, ubest);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  FR_CUDA(cudaGetLastError());
  FR_CUDA(cudaStreamSynchronize(st));
  drop_graphs(s);
  if (out4) {
    Tile tg = R->grad_tile(gbest), tu = R->update_tile(ubest);
    out4[0] = tg.epb; out4[1] = tg.nt; out4[2] = tu.epb; out4[3] = tu.nt;
  }
  return FR_OK;
}

fr_status fr_solver_tile_count(const fr_solver* s, int out2[2])
{
  if (!s || !out2) return fail(FR_ERR_ARG, "bad argument");
  out2[0] = s->run->n_grad_tiles();
  out2[1] = s->run->n_update_tiles();
  return FR_OK;
}

fr_status fr_solver_tile_info(const fr_solver* s, int kind, int i, int out4[4])
{
  if (!s || !out4 || (kind != 0 && kind != 1)) return fail(FR_ERR_ARG, "bad argument");
  const int n = kind == 0 ? s->run->n_grad_tiles() : s->run->n_update_tiles();
  if (i < 0 || i >= n) return fail(FR_ERR_ARG, "tile index out of range");
  const Tile t = kind == 0 ? s->run->grad_tile(i) : s->run->update_tile(i);
  out4[0] = t.epb; out4[1] = t.nt; out4[2] = t.minb; out4[3] = t.pers;
  return FR_OK;
}

fr_status fr_solver_select_tiles(fr_solver* s, int g, int u)
{
  if (!s) return fail(FR_ERR_ARG, "bad argument");
  if (g < 0 || g >= s->run->n_grad_tiles() || u < 0 || u >= s->run->n_update_tiles())
    return fail(FR_ERR_ARG, "tile index out of range");
  FR_CUDA(cudaSetDevice(s->device));
  FR_CUDA(cudaStreamSynchronize(s->own_stream));
  s->run->select(g, u);
  drop_graphs(s);
  return FR_OK;
}

fr_status fr_mesh_geometry(const fr_mesh_desc* md, const fr_scheme_desc* sd, int out6[6], double* pos_upts,
                           double* detjac, double* JG, double* tdA, double* nrm, int* left_idx, int* right_idx)
{
  g_err.clear();
  if (!md || !sd || !out6) return fail(FR_ERR_ARG, "null argument");
  Line1D line;
  Mesh m;
  std::string err;
  if (!make_line(sd->order, sd->upts_type, sd->vcjh_scheme, sd->eta, line, err)) return fail(FR_ERR_ARG, err);
  if (!build_mesh(md->dims, line, md->n_verts, md->xv, md->n_eles, md->c2v, md->shift, md->bctype, m, err))
    return fail(FR_ERR_MESH, err);
  out6[0] = (int)m.ne; out6[1] = m.nu; out6[2] = m.nf; out6[3] = m.nfields; out6[4] = m.dims;
  out6[5] = (int)m.il.size();
  if (pos_upts) memcpy(pos_upts, m.pos_upts.data(), m.pos_upts.size() * 8);
  if (detjac) memcpy(detjac, m.detjac.data(), m.detjac.size() * 8);
  if (JG) memcpy(JG, m.JG.data(), m.JG.size() * 8);
  if (tdA) memcpy(tdA, m.tdA.data(), m.tdA.size() * 8);
  if (nrm) memcpy(nrm, m.nrm.data(), m.nrm.size() * 8);
  if (left_idx) memcpy(left_idx, m.il.data(), m.il.size() * sizeof(int));
  if (right_idx) memcpy(right_idx, m.ir.data(), m.ir.size() * sizeof(int));
  return FR_OK;
}

fr_status fr_line_operators(int order, int upts_type, int vcjh_scheme, double eta, double* out)
{
  if (!out) return fail(FR_ERR_ARG, "null argument");
  Line1D L;
  std::string err;
  if (!make_line(order, upts_type, vcjh_scheme, eta, L, err)) return fail(FR_ERR_ARG, err);
  int n = L.n1;
  double* o = out;
  for (int i = 0; i < n; i++) *o++ = L.loc[i];
  for (int i = 0; i < n; i++) *o++ = L.Lm[i];
  for (int i = 0; i < n; i++) *o++ = L.Lp[i];
  for (int k = 0; k < n; k++) for (int m = 0; m < n; m++) *o++ = L.D[k][m];
  for (int i = 0; i < n; i++) *o++ = L.gL[i];
  for (int i = 0; i < n; i++) *o++ = L.gR[i];
  for (int i = 0; i < n; i++) *o++ = L.w[i];
  *o = L.eta;
  return FR_OK;
}

fr_status fr_solver_sync(fr_solver* s)
{
  if (!s) return fail(FR_ERR_ARG, "null solver");
  FR_CUDA(cudaSetDevice(s->device));
  FR_CUDA(cudaStreamSynchronize(s->own_stream));
  return check_device_flag(s, s->own_stream);
}

}  // extern "C"

fr_status fr_solver_gradient(fr_solver* s, double* host_grad, void* stream)
{
  if (!s || !host_grad) return fail(FR_ERR_ARG, "null argument");
  if (!s->sch.viscous) return fail(FR_ERR_UNSUPPORTED, "the gradient is evaluated on the viscous path only");
  FR_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = STRM(s, stream);
  const Mesh& m = s->mesh;
  const size_t n = (size_t)m.nu * m.ne * m.nfields * m.dims;
  if (!s->grad_buf) {
    char* p;
    fr_status r = dalloc(s, &p, n * s->tc_size);
    if (r) return r;
    s->grad_buf = p;
  }
  Bufs b = s->b;
  b.GRAD = s->grad_buf;
  s->run->grad(b, s->cur, st);
  s->launches++;
  fr_status r = check_launch("fr gradient kernel");
  if (r) return r;
  if (s->tc_size == 8) {
    FR_CUDA(cudaMemcpyAsync(host_grad, s->grad_buf, n * 8, cudaMemcpyDeviceToHost, st));
    FR_CUDA(cudaStreamSynchronize(st));
  } else {
    std::vector<float> f(n);
    FR_CUDA(cudaMemcpyAsync(f.data(), s->grad_buf, n * 4, cudaMemcpyDeviceToHost, st));
    FR_CUDA(cudaStreamSynchronize(st));
    for (size_t i = 0; i < n; i++) host_grad[i] = f[i];
  }
  return FR_OK;
}

fr_status fr_solver_integral_quantities(fr_solver* s, double out5[5], void* stream)
{
  if (!s || !out5) return fail(FR_ERR_ARG, "null argument");
  if (!s->sch.viscous) return fail(FR_ERR_UNSUPPORTED, "the integral quantities need the gradient: viscous path only");
  FR_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = STRM(s, stream);
  const Mesh& m = s->mesh;
  fr_status r = volume_cubature_ready(s);
  if (r) return r;
  const size_t n = (size_t)m.nu * m.ne * m.nfields * m.dims;
  if (!s->grad_buf) {
    char* p;
    if ((r = dalloc(s, &p, n * s->tc_size))) return r;
    s->grad_buf = p;
  }
  Bufs b = s->b;
  b.GRAD = s->grad_buf;
  s->run->grad(b, s->cur, st);
  FR_CUDA(launch_diagnostics(m.dims, (int)s->tc_size, s->b.U, s->grad_buf, s->vc_opp, s->vc_wd, s->vc_detj, m.ne,
                             m.nu, s->vc_n, s->sch.gamma, s->diag_partial, kDiagBlocks, s->diag_out, st));
  s->launches += 3;
  FR_CUDA(cudaMemcpyAsync(out5, s->diag_out, 5 * 8, cudaMemcpyDeviceToHost, st));
  FR_CUDA(cudaStreamSynchronize(st));
  return FR_OK;
}

fr_status fr_solver_sgs_features(fr_solver* s, float* host_x, void* stream)
{
  if (!s || !host_x) return fail(FR_ERR_ARG, "null argument");
  if (!s->sch.viscous) return fail(FR_ERR_UNSUPPORTED, "the closure inputs need the viscous path");
  const Mesh& m = s->mesh;
  const size_t npts = (size_t)m.nu * m.ne;
  std::vector<double> tmp((size_t)npts * m.nfields * m.dims);
  fr_status r = fr_solver_gradient(s, tmp.data(), stream);   // leaves the gradient in grad_buf
  if (r) return r;
  cudaStream_t st = STRM(s, stream);
  if (!s->feat_buf) {
    r = dalloc(s, &s->feat_buf, npts * kMlpIn);
    if (r) return r;
  }
  const double fr = s->sch.les ? s->sch.filter_ratio : 1.0;
  FR_CUDA(launch_sgs_inputs(m.dims, (int)s->tc_size, s->b.U, s->grad_buf, s->b.detj64, (long long)npts, m.nu,
                            (long long)m.ne, s->sch.order, fr, s->feat_buf, st));
  s->launches++;
  FR_CUDA(cudaMemcpyAsync(host_x, s->feat_buf, npts * kMlpIn * sizeof(float), cudaMemcpyDeviceToHost, st));
  FR_CUDA(cudaStreamSynchronize(st));
  return FR_OK;
}

fr_status fr_solver_set_sgs_mlp(fr_solver* s, const float* host_w)
{
  if (!s || !host_w) return fail(FR_ERR_ARG, "null argument");
  if (!s->mlp) return fail(FR_ERR_ARG, "the solver was not created with les = 1, sgs_model = 5");
  for (int p = 0; p < kMlpN; p++)
    if (!std::isfinite(host_w[p])) return fail(FR_ERR_NONFINITE, "non-finite closure parameter");
  FR_CUDA(cudaSetDevice(s->device));
  FR_CUDA(cudaMemcpy(s->mlp, host_w, sizeof(float) * kMlpN, cudaMemcpyHostToDevice));
  return FR_OK;
}

fr_status fr_solver_write_restart(fr_solver* s, const char* path, double time)
{
  if (!s || !path) return fail(FR_ERR_ARG, "null argument");
  const Mesh& m = s->mesh;
  std::vector<double> u((size_t)m.nu * m.ne * m.nfields);
  fr_status r = fr_solver_get_state(s, u.data(), nullptr);
  if (r) return r;
  fr_restart_block b{m.dims == 2 ? 1 : 4, s->sch.order, m.nu, (int)m.ne, m.nfields, s->line.loc, nullptr, u.data(), nullptr};
  return fr_restart_write(path, time, &b, 1);
}

fr_status fr_solver_read_restart(fr_solver* s, const char* path, double* time_out)
{
  if (!s || !path) return fail(FR_ERR_ARG, "null argument");
  const Mesh& m = s->mesh;
  std::vector<double> u((size_t)m.nu * m.ne * m.nfields);
  fr_status r = fr_restart_read(path, m.dims == 2 ? 1 : 4, s->sch.order, s->sch.upts_type, (int)m.ne, m.nfields,
                                nullptr, u.data(), time_out);
  if (r) return r;
  return fr_solver_set_state(s, u.data(), nullptr);
}

// ---------------------------------------------------------------------------
// Batches of independent meshes.  Instances with the same element type,
// order and scheme are merged into one mesh (elements, flux-point indices and
// boundary lists offset; each instance keeps its own periodic wiring), so a
// group is one solver: one launch per stage kernel over all its instances.
// A step of the whole batch (every group, five stages) is one CUDA graph.

namespace {

template <typename V>
void cat_blocks(V& out, const std::vector<const V*>& parts, const std::vector<size_t>& per_elem, int nblocks)
{
  // arrays laid out (n, ne, blocks): per block, the instances' runs one after the other
  out.clear();
  for (int d = 0; d < nblocks; d++)
    for (size_t i = 0; i < parts.size(); i++) {
      const V& a = *parts[i];
      size_t len = a.size() / nblocks;
      out.insert(out.end(), a.begin() + d * len, a.begin() + (d + 1) * len);
    }
  (void)per_elem;
}

bool merge_meshes(std::vector<Mesh>& parts, Mesh& m, std::string& err)
{
  const Mesh& p0 = parts[0];
  m = Mesh();
  m.dims = p0.dims; m.P = p0.P; m.n1 = p0.n1; m.nu = p0.nu; m.nf = p0.nf; m.nface = p0.nface;
  m.nfpf = p0.nfpf; m.nfields = p0.nfields;
  long long ne = 0, nv = 0, nb = 0;
  for (auto& p : parts) ne += p.ne;
  if ((double)m.nf * (double)ne >= 2147483647.0) { err = "batch group too large for 32-bit flux-point indices"; return false; }
  m.ne = ne;
  const int D = m.dims, ns = 1 << D, nf = m.nf;
  std::vector<const std::vector<double>*> pu, pf, dj, jg, ta, nr, nl;
  std::vector<const std::vector<unsigned char>*> il;
  for (auto& p : parts) {
    pu.push_back(&p.pos_upts); pf.push_back(&p.pos_fpts); dj.push_back(&p.detjac); jg.push_back(&p.JG);
    ta.push_back(&p.tdA); nr.push_back(&p.nrm); nl.push_back(&p.nL); il.push_back(&p.is_left);
  }
  std::vector<size_t> none;
  cat_blocks(m.pos_upts, pu, none, D);
  cat_blocks(m.pos_fpts, pf, none, D);
  cat_blocks(m.detjac, dj, none, 1);
  cat_blocks(m.JG, jg, none, 1);
  cat_blocks(m.tdA, ta, none, 1);
  cat_blocks(m.nrm, nr, none, D);
  cat_blocks(m.nL, nl, none, D);
  cat_blocks(m.is_left, il, none, 1);
  long long eoff = 0;
  for (auto& p : parts) {
    const long long fo = (long long)nf * eoff;
    m.xv.insert(m.xv.end(), p.xv.begin(), p.xv.end());
    for (int v : p.c2v) m.c2v.push_back((int)(v + nv));
    for (size_t i = 0; i < p.il.size(); i++) { m.il.push_back((int)(p.il[i] + fo)); m.ir.push_back((int)(p.ir[i] + fo)); }
    for (int q : p.mate) m.mate.push_back(q >= 0 ? (int)(q + fo) : (int)(q - nb));
    for (size_t j = 0; j < p.bf.size(); j++) { m.bf.push_back((int)(p.bf[j] + fo)); m.bt.push_back(p.bt[j]); }
    nv += (long long)(p.xv.size() / D);
    nb += (long long)p.bf.size();
    eoff += p.ne;
  }
  (void)ns;
  return true;
}

bool same_scheme(const fr_scheme_desc& a, const fr_scheme_desc& b)
{
  if (a.order != b.order || a.upts_type != b.upts_type || a.vcjh_scheme != b.vcjh_scheme || a.eta != b.eta ||
      a.viscous != b.viscous || a.riemann != b.riemann || a.precision != b.precision || a.gamma != b.gamma ||
      a.prandtl != b.prandtl || a.mu_inf != b.mu_inf || a.rt_inf != b.rt_inf || a.c_sth != b.c_sth ||
      a.fix_vis != b.fix_vis || a.tau != b.tau || a.pen_fact != b.pen_fact || a.les != b.les ||
      a.sgs_model != b.sgs_model || a.filter_ratio != b.filter_ratio || a.R_ref != b.R_ref)
    return false;
  for (int i = 0; i < 14; i++)
    if (a.bdy[i] != b.bdy[i]) return false;
  return true;
}

}  // namespace

struct fr_batch {
  int device = 0;
  std::vector<fr_solver*> groups;
  std::vector<int> inst_group;            // instance -> group
  std::vector<long long> inst_eoff, inst_ne;
  std::vector<char> dirty;                // group state written since its traces were made
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  double graph_dt[2] = {0, 0};
  long long launches = 0;
  int merged = 0;                         // 1: one launch per stage kernel for all groups
  int merged_minb = 4;                    // CTAs per SM the merged kernels' registers are capped for
};

namespace {

// One stage of every group as merged launches (fr_batch_merged.cuh).
template <typename TC>
fr_status merged_stage_t(fr_batch* b, int k, double dt, cudaStream_t st)
{
  MergedGrads<TC> G{};
  MergedFaces<TC> Fc{};
  MergedUpds<TC> U{};
  bool any_face = false;
  for (fr_solver* s : b->groups) {
    MergedGrad<TC> g{};
    MergedFace<TC> f{};
    MergedUpd<TC> u{};
    int P = s->run->merged_args(s->b, s->cur, k, dt, &g, &f, &u);
    if (P < 2 || P > 4) return fail(FR_ERR_UNSUPPORTED, "a group cannot join the merged launches");
    G.s[P - 2] = g;
    Fc.s[P - 2] = f;
    U.s[P - 2] = u;
    any_face = any_face || f.nblk > 0;
  }
  fr_status r = merged_stage_launch(sizeof(TC) == 4, &G, &Fc, any_face, &U, b->merged_minb, st);
  for (fr_solver* s : b->groups) s->cur ^= 1;
  return r;
}

// Groups that can run merged: hexahedra of orders 2-4, at most one group per
// order, all viscous without LES, Rusanov, one precision.
bool batch_mergeable(const fr_batch* b, std::string& why)
{
  int seen[5] = {0, 0, 0, 0, 0};
  for (const fr_solver* s : b->groups) {
    const fr_scheme_desc& d = s->sch;
    if (s->mesh.dims != 3 || d.order < 2 || d.order > 4) { why = "merged launches take hexahedra of orders 2-4"; return false; }
    if (seen[d.order]++) { why = "merged launches take one group per order"; return false; }
    if (!d.viscous || d.les || d.riemann != 0) { why = "merged launches take viscous Rusanov groups without LES"; return false; }
    if (d.precision != b->groups[0]->sch.precision) { why = "merged launches take one precision"; return false; }
  }
  return true;
}

}  // namespace

extern "C" {

fr_status fr_batch_destroy(fr_batch* b)
{
  if (!b) return FR_OK;
  cudaSetDevice(b->device);
  for (int i = 0; i < 2; i++)
    if (b->graph[i]) cudaGraphExecDestroy(b->graph[i]);
  if (b->stream) { cudaStreamSynchronize(b->stream); cudaStreamDestroy(b->stream); }
  for (fr_solver* s : b->groups) fr_solver_destroy(s);
  delete b;
  return FR_OK;
}

fr_status fr_batch_create(const fr_mesh_desc* meshes, const fr_scheme_desc* schemes, int n, int device,
                          fr_batch** out)
{
  g_err.clear();
  if (!meshes || !schemes || !out || n < 1) return fail(FR_ERR_ARG, "bad argument");
  *out = nullptr;
  std::unique_ptr<fr_batch, fr_status (*)(fr_batch*)> b(new fr_batch(), fr_batch_destroy);
  b->device = device;
  b->inst_group.assign(n, -1);
  b->inst_eoff.assign(n, 0);
  b->inst_ne.assign(n, 0);
  std::vector<int> done(n, 0);
  for (int i = 0; i < n; i++) {
    if (done[i]) continue;
    std::vector<int> members;
    for (int j = i; j < n; j++)
      if (!done[j] && meshes[j].dims == meshes[i].dims && same_scheme(schemes[j], schemes[i])) {
        members.push_back(j);
        done[j] = 1;
      }
    const fr_scheme_desc* sd = &schemes[i];
    fr_status v = validate_scheme(meshes[i].dims, sd);
    if (v) return v;
    Line1D line;
    std::string err;
    if (!make_line(sd->order, sd->upts_type, sd->vcjh_scheme, sd->eta, line, err)) return fail(FR_ERR_ARG, err);
    std::vector<Mesh> parts(members.size());
    long long eoff = 0;
    for (size_t q = 0; q < members.size(); q++) {
      const fr_mesh_desc* md = &meshes[members[q]];
      if (!build_mesh(md->dims, line, md->n_verts, md->xv, md->n_eles, md->c2v, md->shift, md->bctype, parts[q],
                      err))
        return fail(FR_ERR_MESH, "instance " + std::to_string(members[q]) + ": " + err);
      b->inst_group[members[q]] = (int)b->groups.size();
      b->inst_eoff[members[q]] = eoff;
      b->inst_ne[members[q]] = parts[q].ne;
      eoff += parts[q].ne;
    }
    Mesh merged;
    if (!merge_meshes(parts, merged, err)) return fail(FR_ERR_MESH, err);
    parts.clear();
    fr_solver* s = nullptr;
    // validation of the scheme (orders, models) is fr_solver_create's: run it on the first instance's shape
    fr_status st = create_with_mesh(std::move(merged), line, sd, device, &s);
    if (st) return st;
    b->groups.push_back(s);
  }
  b->dirty.assign(b->groups.size(), 1);
  FR_CUDA(cudaSetDevice(device));
  FR_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  *out = b.release();
  return FR_OK;
}

int fr_batch_n_groups(const fr_batch* b) { return b ? (int)b->groups.size() : 0; }

fr_status fr_batch_group(fr_batch* b, int g, fr_solver** out)
{
  if (!b || !out || g < 0 || g >= (int)b->groups.size()) return fail(FR_ERR_ARG, "bad group");
  *out = b->groups[g];
  return FR_OK;
}

fr_status fr_batch_instance(const fr_batch* b, int i, int out4[4])
{
  if (!b || !out4 || i < 0 || i >= (int)b->inst_group.size()) return fail(FR_ERR_ARG, "bad instance");
  const fr_solver* s = b->groups[b->inst_group[i]];
  out4[0] = b->inst_group[i];
  out4[1] = (int)b->inst_eoff[i];
  out4[2] = (int)b->inst_ne[i];
  out4[3] = s->mesh.nu;
  return FR_OK;
}

fr_status fr_batch_set_state(fr_batch* b, int i, const double* host_u)
{
  if (!b || !host_u || i < 0 || i >= (int)b->inst_group.size()) return fail(FR_ERR_ARG, "bad argument");
  const int g = b->inst_group[i];
  fr_solver* s = b->groups[g];
  const size_t nu = s->mesh.nu, E = s->mesh.ne, F = s->mesh.nfields, ne = b->inst_ne[i], eo = b->inst_eoff[i];
  for (size_t q = 0; q < nu * ne * F; q++)
    if (!std::isfinite(host_u[q])) return fail(FR_ERR_NONFINITE, "non-finite state");
  FR_CUDA(cudaSetDevice(b->device));
  for (size_t k = 0; k < F; k++) {
    FR_CUDA(cudaMemcpyAsync(s->b.U + nu * (eo + E * k), host_u + nu * ne * k, nu * ne * 8, cudaMemcpyHostToDevice,
                            b->stream));
    FR_CUDA(cudaMemsetAsync(s->b.REG + nu * (eo + E * k), 0, nu * ne * 8, b->stream));
  }
  FR_CUDA(cudaStreamSynchronize(b->stream));
  b->dirty[g] = 1;
  return FR_OK;
}

fr_status fr_batch_get_state(fr_batch* b, int i, double* host_u)
{
  if (!b || !host_u || i < 0 || i >= (int)b->inst_group.size()) return fail(FR_ERR_ARG, "bad argument");
  fr_solver* s = b->groups[b->inst_group[i]];
  const size_t nu = s->mesh.nu, E = s->mesh.ne, F = s->mesh.nfields, ne = b->inst_ne[i], eo = b->inst_eoff[i];
  FR_CUDA(cudaSetDevice(b->device));
  for (size_t k = 0; k < F; k++)
    FR_CUDA(cudaMemcpyAsync(host_u + nu * ne * k, s->b.U + nu * (eo + E * k), nu * ne * 8, cudaMemcpyDeviceToHost,
                            b->stream));
  FR_CUDA(cudaStreamSynchronize(b->stream));
  return FR_OK;
}

fr_status fr_batch_autotune(fr_batch* b, int reps)
{
  if (!b) return fail(FR_ERR_ARG, "null batch");
  int t[4];
  for (size_t g = 0; g < b->groups.size(); g++) {
    fr_status st = fr_solver_state_updated(b->groups[g], b->stream);
    if (st) return st;
    b->dirty[g] = 0;
    st = fr_solver_autotune(b->groups[g], reps, t);
    if (st) return st;
  }
  for (int i = 0; i < 2; i++)
    if (b->graph[i]) { cudaGraphExecDestroy(b->graph[i]); b->graph[i] = nullptr; }
  // per-group graph against merged launches (two register caps): time `reps`
  // whole steps of each from the same state, restore the state after each
  std::string why;
  b->merged = 0;
  if (!batch_mergeable(b, why)) return FR_OK;
  FR_CUDA(cudaSetDevice(b->device));
  std::vector<double*> saved(b->groups.size(), nullptr);
  fr_status r = FR_OK;
  for (size_t g = 0; g < b->groups.size() && r == FR_OK; g++) {
    fr_solver* s = b->groups[g];
    size_t bytes = sizeof(double) * (size_t)s->mesh.nu * s->mesh.ne * s->mesh.nfields;
    if (cudaMalloc(&saved[g], bytes) != cudaSuccess) { saved[g] = nullptr; r = fail(FR_ERR_CUDA, "autotune state copy"); break; }
    if (cudaMemcpyAsync(saved[g], s->b.U, bytes, cudaMemcpyDeviceToDevice, b->stream) != cudaSuccess)
      r = fail(FR_ERR_CUDA, "autotune state copy");
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double best = 1e30;
  int best_mode = 0, best_minb = 4;
  const int modes[3][2] = {{0, 4}, {1, 4}, {1, 3}};
  if (r == FR_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    r = fail(FR_ERR_CUDA, "autotune events");
  for (int m = 0; m < 3 && r == FR_OK; m++) {
    b->merged = modes[m][0];
    b->merged_minb = modes[m][1];
    for (int i = 0; i < 2; i++)
      if (b->graph[i]) { cudaGraphExecDestroy(b->graph[i]); b->graph[i] = nullptr; }
    const double dt = 1e-5;
    r = fr_batch_advance(b, 2, dt, b->stream);                   // capture both graphs, warm up
    if (r == FR_OK) cudaEventRecord(e0, b->stream);
    if (r == FR_OK) r = fr_batch_advance(b, reps, dt, b->stream);
    if (r == FR_OK) cudaEventRecord(e1, b->stream);
    if (r == FR_OK && cudaEventSynchronize(e1) != cudaSuccess) r = fail(FR_ERR_CUDA, "autotune timing");
    float ms = 0.f;
    if (r == FR_OK) cudaEventElapsedTime(&ms, e0, e1);
    if (r == FR_OK && ms < best) { best = ms; best_mode = modes[m][0]; best_minb = modes[m][1]; }
    // back to the saved state (traces rebuilt from it)
    for (size_t g = 0; g < b->groups.size() && r == FR_OK; g++) {
      fr_solver* s = b->groups[g];
      size_t bytes = sizeof(double) * (size_t)s->mesh.nu * s->mesh.ne * s->mesh.nfields;
      if (cudaMemcpyAsync(s->b.U, saved[g], bytes, cudaMemcpyDeviceToDevice, b->stream) != cudaSuccess)
        r = fail(FR_ERR_CUDA, "autotune state restore");
      if (r == FR_OK) r = fr_solver_state_updated(s, b->stream);
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaStreamSynchronize(b->stream);
  for (double* p : saved)
    if (p) cudaFree(p);
  b->merged = r == FR_OK ? best_mode : 0;
  b->merged_minb = best_minb;
  for (int i = 0; i < 2; i++)
    if (b->graph[i]) { cudaGraphExecDestroy(b->graph[i]); b->graph[i] = nullptr; }
  return r;
}

fr_status fr_batch_set_merged(fr_batch* b, int on, int minb)
{
  if (!b) return fail(FR_ERR_ARG, "null batch");
  std::string why;
  if (on && !batch_mergeable(b, why)) return fail(FR_ERR_UNSUPPORTED, why);
  if (on && minb != 1 && minb != 3 && minb != 4) return fail(FR_ERR_ARG, "minb must be 1, 3 or 4");
  b->merged = on ? 1 : 0;
  if (on) b->merged_minb = minb;
  for (int i = 0; i < 2; i++)
    if (b->graph[i]) { cudaGraphExecDestroy(b->graph[i]); b->graph[i] = nullptr; }
  return FR_OK;
}

int fr_batch_merged(const fr_batch* b) { return b && b->merged ? b->merged_minb : 0; }

fr_status fr_batch_advance(fr_batch* b, int n_steps, double dt, void* stream)
{
  if (!b || n_steps < 0) return fail(FR_ERR_ARG, "bad argument");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(FR_ERR_ARG, "dt must be positive");
  FR_CUDA(cudaSetDevice(b->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
  for (size_t g = 0; g < b->groups.size(); g++)
    if (b->dirty[g]) {
      fr_status r = fr_solver_state_updated(b->groups[g], st);
      if (r) return r;
      b->dirty[g] = 0;
    }
  const int c0 = b->groups[0]->cur;
  for (fr_solver* s : b->groups)
    if (s->cur != c0) return fail(FR_ERR_ARG, "groups out of step");
  long long per_step = 0;
  if (b->merged) {
    bool any_face = false;
    for (fr_solver* s : b->groups) any_face = any_face || s->run->launches_per_stage() == 3;
    per_step = 5 * (any_face ? 3 : 2);
  } else {
    for (fr_solver* s : b->groups) per_step += 5 * s->run->launches_per_stage();
  }
  for (int i = 0; i < n_steps; i++) {
    const int c = b->groups[0]->cur;
    if (!b->graph[c] || b->graph_dt[c] != dt) {
      if (b->graph[c]) { cudaGraphExecDestroy(b->graph[c]); b->graph[c] = nullptr; }
      cudaGraph_t gr;
      FR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      fr_status cr = FR_OK;
      for (int k = 0; k < 5 && cr == FR_OK; k++) {
        if (b->merged) {
          cr = b->groups[0]->sch.precision == 1 ? merged_stage_t<float>(b, k, dt, st) : merged_stage_t<double>(b, k, dt, st);
          continue;
        }
        for (fr_solver* s : b->groups) {
          long long l0 = s->launches;
          stage(s, k, dt, k == 4, st);
          s->launches = l0;
        }
      }
      for (fr_solver* s : b->groups) s->cur = c;
      FR_CUDA(cudaStreamEndCapture(st, &gr));
      if (cr) { cudaGraphDestroy(gr); return cr; }
      cudaError_t e = cudaGraphInstantiate(&b->graph[c], gr, 0);
      cudaGraphDestroy(gr);
      if (e != cudaSuccess) return fail(FR_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      b->graph_dt[c] = dt;
    }
    FR_CUDA(cudaGraphLaunch(b->graph[c], st));
    b->launches += per_step;
    for (fr_solver* s : b->groups) s->cur ^= 1;
  }
  return FR_OK;
}

long long fr_batch_launch_count(const fr_batch* b) { return b ? b->launches : 0; }
void* fr_batch_stream(fr_batch* b) { return b ? (void*)b->stream : nullptr; }

}  // extern "C"

extern "C" fr_status fr_solver_write_vtu(fr_solver* s, const char* path)
{
  if (!s || !path) return fail(FR_ERR_ARG, "null argument");
  const Mesh& m = s->mesh;
  std::vector<double> u((size_t)m.nu * m.ne * m.nfields);
  fr_status r = fr_solver_get_state(s, u.data(), nullptr);
  if (r) return r;
  return fr_vtu_write(path, m.dims, s->sch.order, (int)m.ne, m.pos_upts.data(), u.data(), s->sch.gamma);
}
