// pybind11 module _gs2g: a thin Python binding of the C-ABI in include/gs2g.h.
// It converts numpy arrays to plain pointers and C status codes to Python
// exceptions (GS2G_ERR_INVALID -> ValueError, others -> RuntimeError), the
// error mapping of the reference's pybind11 module (src/_cpp/python_bindings.cpp).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/gs2g.h"

namespace py = pybind11;

namespace {

// ---- DLPack export -----------------------------------------------------
// The DLPack ABI (dlpack.h v0.8 layout), written out here: device buffers of
// the session are exported zero-copy, as the reference's v_results_dlpack
// (src/_cpp/dlpack_export.hpp:20-45).  The capsule aliases live device memory
// and stays valid until the next run on the same session.
struct DLDevice_ {
  int32_t device_type;
  int32_t device_id;
};
struct DLDataType_ {
  uint8_t code;
  uint8_t bits;
  uint16_t lanes;
};
struct DLTensor_ {
  void* data;
  DLDevice_ device;
  int32_t ndim;
  DLDataType_ dtype;
  int64_t* shape;
  int64_t* strides;
  uint64_t byte_offset;
};
struct DLManagedTensor_ {
  DLTensor_ dl_tensor;
  void* manager_ctx;
  void (*deleter)(DLManagedTensor_*);
};
struct DLCtx {
  int64_t shape[2];
};
enum : int32_t { kDLCUDA_ = 2 };
enum : uint8_t { kDLInt_ = 0, kDLFloat_ = 2, kDLComplex_ = 5 };

void dl_deleter(DLManagedTensor_* t) {
  delete static_cast<DLCtx*>(t->manager_ctx);
  delete t;
}

py::capsule make_dlpack(void* ptr, int device, int ndim, int64_t d0, int64_t d1, uint8_t code, uint8_t bits) {
  auto* ctx = new DLCtx{{d0, d1}};
  auto* t = new DLManagedTensor_{};
  t->dl_tensor.data = ptr;
  t->dl_tensor.device = {kDLCUDA_, device};
  t->dl_tensor.ndim = ndim;
  t->dl_tensor.dtype = {code, bits, 1};
  t->dl_tensor.shape = ctx->shape;
  t->dl_tensor.strides = nullptr;
  t->dl_tensor.byte_offset = 0;
  t->manager_ctx = ctx;
  t->deleter = dl_deleter;
  return py::capsule(t, "dltensor", [](PyObject* cap) {
    // a consumed capsule is renamed "used_dltensor" and owned by its consumer
    if (PyCapsule_IsValid(cap, "dltensor")) {
      auto* m = static_cast<DLManagedTensor_*>(PyCapsule_GetPointer(cap, "dltensor"));
      if (m && m->deleter) m->deleter(m);
    }
  });
}

using cplx = std::complex<double>;
using IArr = py::array_t<int, py::array::c_style | py::array::forcecast>;
using DArr = py::array_t<double, py::array::c_style | py::array::forcecast>;
using CArr = py::array_t<cplx, py::array::c_style | py::array::forcecast>;

void check(int rc) {
  if (rc == GS2G_OK) return;
  std::string msg = gs2g_last_error();
  if (rc == GS2G_ERR_INVALID) throw py::value_error(msg);
  throw std::runtime_error(msg);
}

gs2g_run_opts make_opts(int max_iter, double tol, bool fixed_iters, int precision, int start, double pivot_floor,
                        int n_ctas, bool profile = false, int refactor = 0, double refactor_ratio = 0.0,
                        int max_reuse = 0, bool rescue = false, int iters_per_round = 1,
                        bool step_then_check = false, bool step_scaling = false, double max_dva = 0.0,
                        double max_dvm = 0.0) {
  gs2g_run_opts o{};
  o.max_iter = max_iter;
  o.tol = tol;
  o.fixed_iters = fixed_iters ? 1 : 0;
  o.precision = precision;
  o.start = start;
  o.pivot_floor = pivot_floor;
  o.n_ctas = n_ctas;
  o.profile_phases = profile ? 1 : 0;
  o.refactor_policy = refactor;
  o.refactor_ratio = refactor_ratio;
  o.max_reuse = max_reuse;
  o.rescue = rescue ? 1 : 0;
  o.iters_per_round = iters_per_round;
  o.step_then_check = step_then_check ? 1 : 0;
  o.step_scaling = step_scaling ? 1 : 0;
  o.max_dva = max_dva;
  o.max_dvm = max_dvm;
  return o;
}

class Session {
 public:
  Session(int device, int n_bus, IArr indptr, IArr indices, CArr data, CArr vinit, CArr sbus, IArr pv, IArr pq,
          int tail_policy)
      : n_bus_(n_bus) {
    if (indptr.size() != n_bus + 1) throw py::value_error("Ybus indptr must have n_bus + 1 entries");
    if (indices.size() != data.size()) throw py::value_error("Ybus indices and data differ in length");
    if (vinit.size() != n_bus || sbus.size() != n_bus) throw py::value_error("Vinit and Sbus must have n_bus entries");
    if (indptr.at(n_bus) != indices.size()) throw py::value_error("Ybus indptr[-1] must equal nnz");
    const double* dv = reinterpret_cast<const double*>(data.data());
    int rc;
    {
      py::gil_scoped_release nogil;
      rc = gs2g_session_create(device, n_bus, indptr.data(), indices.data(), dv,
                               reinterpret_cast<const double*>(vinit.data()),
                               reinterpret_cast<const double*>(sbus.data()), pv.data(), (int)pv.size(), pq.data(),
                               (int)pq.size(), tail_policy, &s_);
    }
    check(rc);
  }
  ~Session() {
    if (s_) gs2g_session_destroy(s_);
  }
  void close() {
    if (s_) gs2g_session_destroy(s_);
    s_ = nullptr;
  }
  gs2g_session* h() const {
    if (!s_) throw std::runtime_error("session is closed");
    return s_;
  }
  // the C-ABI handle, for callers that drive include/gs2g.h directly
  uintptr_t handle() const { return reinterpret_cast<uintptr_t>(h()); }

  py::dict info() const {
    gs2g_grid_info g{};
    check(gs2g_grid_get_info(h(), &g));
    py::dict d;
    d["n_bus"] = g.n_bus;
    d["nnz_y"] = g.nnz_y;
    d["n_pvpq"] = g.n_pvpq;
    d["n_pq"] = g.n_pq;
    d["dim_j"] = g.dim_j;
    d["nnz_j"] = g.nnz_j;
    d["nnz_lu"] = g.nnz_lu;
    d["head_dim"] = g.head_dim;
    d["tail_dim"] = g.tail_dim;
    d["tail_dim_exact"] = g.tail_dim_exact;
    d["n_levels"] = g.n_levels;
    d["n_supernodes"] = g.n_supernodes;
    d["head_madds"] = g.head_madds;
    d["schur_madds"] = g.schur_madds;
    d["dense_madds"] = g.dense_madds;
    d["plan_ms"] = g.plan_ms;
    return d;
  }

  void set_branch_data(IArr f, IArr t, CArr yff, CArr yft, CArr ytf, CArr ytt) {
    const int nb = (int)f.size();
    if (t.size() != nb || yff.size() != nb || yft.size() != nb || ytf.size() != nb || ytt.size() != nb)
      throw py::value_error("branch arrays differ in length");
    auto d = [](const CArr& a) { return reinterpret_cast<const double*>(a.data()); };
    check(gs2g_set_branch_data(h(), nb, f.data(), t.data(), d(yff), d(yft), d(ytf), d(ytt)));
  }

  void set_contingencies(IArr ptr, IArr ids) {
    const int nr = (int)ptr.size() - 1;
    if (nr < 0) throw py::value_error("ptr must have n_rows + 1 entries");
    check(gs2g_set_contingencies(h(), nr, ptr.data(), ids.data()));
  }

  void clear_contingencies() { check(gs2g_set_contingencies(h(), 0, nullptr, nullptr)); }

  void set_injections(DArr p, DArr q, double sn_mva) {
    if (p.ndim() != 2 || q.ndim() != 2 || p.shape(1) != n_bus_ || q.shape(0) != p.shape(0) || q.shape(1) != n_bus_)
      throw py::value_error("p_mw / q_mvar must both be (n_rows, n_bus)");
    const int nr = (int)p.shape(0);
    int rc;
    {
      py::gil_scoped_release nogil;
      rc = gs2g_set_injections(h(), nr, p.data(), q.data(), sn_mva);
    }
    check(rc);
  }

  void clear_injections() { check(gs2g_set_injections(h(), 0, nullptr, nullptr, 1.0)); }

  void set_start_rows(CArr v0) {
    if (v0.ndim() != 2 || v0.shape(1) != n_bus_) throw py::value_error("start rows must be (n_rows, n_bus) complex");
    check(gs2g_set_start_rows(h(), (int)v0.shape(0), reinterpret_cast<const double*>(v0.data())));
  }

  void set_start_rows_device(uintptr_t ptr, int n_rows) {
    check(gs2g_set_start_rows_device(h(), n_rows, reinterpret_cast<const double*>(ptr)));
  }

  void run_subset(IArr rows, int max_iter, double tol, bool fixed_iters, int precision, int start,
                  double pivot_floor, int n_ctas, int refactor, double refactor_ratio, int max_reuse, bool rescue,
                  int iters_per_round, bool profile, bool step_scaling, double max_dva, double max_dvm) {
    gs2g_run_opts o = make_opts(max_iter, tol, fixed_iters, precision, start, pivot_floor, n_ctas, profile, refactor,
                                refactor_ratio, max_reuse, rescue, iters_per_round, false, step_scaling, max_dva,
                                max_dvm);
    const int n = (int)rows.size();
    const int* rp = rows.data();
    int rc;
    {
      py::gil_scoped_release nogil;
      rc = gs2g_run_subset(h(), &o, n, rp);
    }
    check(rc);
  }

  void replan(int tail_policy, double dense_rate, int force_tau) {
    check(gs2g_session_replan(h(), tail_policy, dense_rate, force_tau));
  }

  void set_chord(int mode) { check(gs2g_session_set_chord(h(), mode)); }
  void set_handoff(int cluster) { check(gs2g_session_set_handoff(h(), cluster)); }
  void set_results_mirror(bool on) { check(gs2g_session_set_results_mirror(h(), on ? 1 : 0)); }
  void set_row_order(bool on) { check(gs2g_session_set_row_order(h(), on ? 1 : 0)); }
  // adjoint: raw device pointers of rhs / lam [n_rows x dim_J] (caller-owned)
  void solve_jt(int n_rows, uintptr_t rhs, uintptr_t lam) {
    int rc;
    {
      py::gil_scoped_release nogil;
      rc = gs2g_solve_jt(h(), n_rows, reinterpret_cast<const double*>(rhs), reinterpret_cast<double*>(lam));
    }
    check(rc);
  }
  void set_handle_disconnected(bool on) { check(gs2g_session_set_handle_disconnected(h(), on ? 1 : 0)); }

  uintptr_t start_rows_buffer(int n_rows) {
    double* p = nullptr;
    check(gs2g_start_rows_buffer(h(), n_rows, &p));
    return reinterpret_cast<uintptr_t>(p);
  }

  void set_sbus(CArr sbus) {
    if (sbus.size() != n_bus_) throw py::value_error("Sbus must have n_bus entries");
    check(gs2g_set_sbus(h(), reinterpret_cast<const double*>(sbus.data())));
  }

  void set_vinit(CArr v) {
    if (v.size() != n_bus_) throw py::value_error("Vinit must have n_bus entries");
    check(gs2g_set_vinit(h(), reinterpret_cast<const double*>(v.data())));
  }

  // the base case is a single solve: the reference's step-then-test order by default
  py::tuple solve_base(int max_iter, double tol, int precision, double pivot_floor, bool step_then_check) {
    gs2g_run_opts o = make_opts(max_iter, tol, false, precision, GS2G_START_VINIT, pivot_floor, 1, false, 0, 0.0, 0,
                                false, 1, step_then_check);
    py::array_t<cplx> V(n_bus_);
    int st = 0, it = 0;
    double res = 0;
    int rc;
    {
      cplx* vp = V.mutable_data();
      py::gil_scoped_release nogil;
      rc = gs2g_solve_base(h(), &o, reinterpret_cast<double*>(vp), &st, &it, &res);
    }
    check(rc);
    return py::make_tuple(V, st, it, res);
  }

  double set_base_v(CArr v) {
    if (v.size() != n_bus_) throw py::value_error("V must have n_bus entries");
    double res = 0;
    check(gs2g_set_base_v(h(), reinterpret_cast<const double*>(v.data()), &res));
    return res;
  }

  void run(int max_iter, double tol, bool fixed_iters, int precision, int start, double pivot_floor, int n_ctas,
           bool profile, int refactor, double refactor_ratio, int max_reuse, bool rescue, int iters_per_round,
           bool step_then_check, bool step_scaling, double max_dva, double max_dvm) {
    gs2g_run_opts o = make_opts(max_iter, tol, fixed_iters, precision, start, pivot_floor, n_ctas, profile, refactor,
                                refactor_ratio, max_reuse, rescue, iters_per_round, step_then_check, step_scaling,
                                max_dva, max_dvm);
    int rc;
    {
      py::gil_scoped_release nogil;
      rc = gs2g_run(h(), &o);
    }
    check(rc);
  }

  int n_rows() const { return gs2g_n_rows(h()); }

  void set_branch_limits(DArr rate_mva, double sn_mva) {
    check(gs2g_set_branch_limits(h(), (int)rate_mva.size(), rate_mva.data(), sn_mva));
  }

  py::tuple branch_loading(int n_branch) const {
    const int nr = gs2g_n_rows(h());
    py::array_t<float> ld({nr, n_branch});
    py::array_t<int> nv(nr);
    py::array_t<float> mx(nr);
    int rc;
    {
      float* lp = ld.mutable_data();
      int* np_ = nv.mutable_data();
      float* mp = mx.mutable_data();
      py::gil_scoped_release nogil;
      rc = gs2g_get_branch_loading(h(), lp, np_, mp);
    }
    check(rc);
    return py::make_tuple(ld, nv, mx);
  }

  py::tuple results() const {
    const int nr = gs2g_n_rows(h());
    py::array_t<cplx> V({nr, n_bus_});
    py::array_t<double> res(nr);
    py::array_t<int> st(nr), it(nr);
    int rc;
    {
      double* vp = reinterpret_cast<double*>(V.mutable_data());
      double* rp = res.mutable_data();
      int* sp = st.mutable_data();
      int* ip = it.mutable_data();
      py::gil_scoped_release nogil;
      rc = gs2g_get_results(h(), vp, rp, sp, ip);
    }
    check(rc);
    return py::make_tuple(V, res, st, it);
  }

  // numpy views of the session's pinned host copy of the last results
  // (gs2g_get_results_host), kept alive by this session object; valid until
  // the next results_view(), run or close
  py::tuple results_view(py::object self) {
    double *v = nullptr, *r = nullptr;
    int *st = nullptr, *it = nullptr;
    int rc;
    {
      py::gil_scoped_release nogil;
      rc = gs2g_get_results_host(h(), &v, &r, &st, &it);
    }
    check(rc);
    const py::ssize_t nr = gs2g_n_rows(h());
    py::array_t<cplx> V({nr, (py::ssize_t)n_bus_}, reinterpret_cast<cplx*>(v), self);
    py::array_t<double> res({nr}, r, self);
    py::array_t<int> sa({nr}, st, self);
    py::array_t<int> ia({nr}, it, self);
    return py::make_tuple(V, res, sa, ia);
  }

  py::array_t<int> factor_counts() const {
    const int nr = gs2g_n_rows(h());
    py::array_t<int> f(nr);
    check(gs2g_get_factor_counts(h(), f.mutable_data()));
    return f;
  }

  py::tuple device_results() const {
    double *v = nullptr, *r = nullptr;
    int *s = nullptr, *i = nullptr;
    check(gs2g_get_device_results(h(), &v, &r, &s, &i));
    return py::make_tuple((uintptr_t)v, (uintptr_t)r, (uintptr_t)s, (uintptr_t)i);
  }

  // DLPack capsules of the last run's device results: "v" (n_rows, n_bus)
  // complex128, "residuals" (n_rows,) float64, "status"/"iters" (n_rows,) int32.
  py::capsule dlpack(const std::string& what) const {
    double *v = nullptr, *r = nullptr;
    int *s = nullptr, *i = nullptr;
    check(gs2g_get_device_results(h(), &v, &r, &s, &i));
    const int nr = gs2g_n_rows(h());
    int dev = 0;
    check(gs2g_get_device(h(), &dev));
    if (what == "v") return make_dlpack(v, dev, 2, nr, n_bus_, kDLComplex_, 128);
    if (what == "residuals") return make_dlpack(r, dev, 1, nr, 0, kDLFloat_, 64);
    if (what == "status") return make_dlpack(s, dev, 1, nr, 0, kDLInt_, 32);
    if (what == "iters") return make_dlpack(i, dev, 1, nr, 0, kDLInt_, 32);
    throw py::value_error("unknown result '" + what + "'");
  }

  // DLPack capsules of the current rows on the device: "sbus" (n_rows, n_bus)
  // complex128, "trip_ptr" (n_rows + 1,) / "trip_ids" (n_ids,) int32; None
  // when the rows have no such definition.
  py::object device_rows(const std::string& what) {
    int nr = 0;
    const double* sb = nullptr;
    const int *tp = nullptr, *ti = nullptr;
    int64_t nid = 0;
    check(gs2g_get_device_rows(h(), &nr, &sb, &tp, &ti, &nid));
    int dev = 0;
    check(gs2g_get_device(h(), &dev));
    if (what == "sbus") return sb ? py::object(make_dlpack(const_cast<double*>(sb), dev, 2, nr, n_bus_, kDLComplex_, 128)) : py::none();
    if (what == "trip_ptr") return tp ? py::object(make_dlpack(const_cast<int*>(tp), dev, 1, nr + 1, 0, kDLInt_, 32)) : py::none();
    if (what == "trip_ids")
      return ti ? py::object(make_dlpack(const_cast<int*>(ti), dev, 1, std::max<int64_t>(nid, 0), 0, kDLInt_, 32))
                : py::none();
    throw py::value_error("unknown row definition '" + what + "'");
  }

  py::dict timings() const {
    gs2g_timings t{};
    check(gs2g_get_timings(h(), &t));
    py::dict d;
    d["plan_ms"] = t.plan_ms;
    d["upload_ms"] = t.upload_ms;
    d["kernel_ms"] = t.kernel_ms;
    d["total_ms"] = t.total_ms;
    d["total_iters"] = t.total_iters;
    py::list pc, ps;
    for (int q = 0; q < GS2G_N_PHASES; ++q) {
      pc.append(t.phase_cycles[q]);
      ps.append(t.phase_share[q]);
    }
    d["phase_cycles"] = pc;
    d["phase_share"] = ps;
    d["n_rescued"] = t.n_rescued;
    d["n_base_start"] = t.n_base_start;
    d["chord_steps"] = t.chord_steps;
    d["base_setup_ms"] = t.base_setup_ms;
    d["base_setup_bytes"] = t.base_setup_bytes;
    d["n_failed"] = t.n_failed;
    return d;
  }

  void sync() { check(gs2g_sync(h())); }
  void wait_stream(uintptr_t stream) { check(gs2g_session_wait_stream(h(), reinterpret_cast<void*>(stream))); }

 private:
  gs2g_session* s_ = nullptr;
  int n_bus_ = 0;
};

py::tuple acpf_nr(int device, int n_bus, IArr indptr, IArr indices, CArr data, CArr V, CArr sbus, IArr pv, IArr pq,
                  int max_iter, double tol, int precision) {
  if (V.size() != n_bus || sbus.size() != n_bus) throw py::value_error("V and Sbus must have n_bus entries");
  py::array_t<cplx> out(n_bus);
  std::memcpy(out.mutable_data(), V.data(), sizeof(cplx) * n_bus);
  int conv = 0, it = 0;
  double res = 0, ms = 0;
  int rc;
  {
    double* op = reinterpret_cast<double*>(out.mutable_data());
    py::gil_scoped_release nogil;
    rc = gs2g_acpf_nr(device, n_bus, indptr.data(), indices.data(), reinterpret_cast<const double*>(data.data()), op,
                      reinterpret_cast<const double*>(sbus.data()), pv.data(), (int)pv.size(), pq.data(),
                      (int)pq.size(), max_iter, tol, precision, &conv, &it, &res, &ms);
  }
  check(rc);
  return py::make_tuple(out, conv != 0, it, res, ms);
}

py::dict plan_info(int n_bus, IArr indptr, IArr indices, IArr pv, IArr pq, int tail_policy) {
  if (indptr.size() != n_bus + 1) throw py::value_error("Ybus indptr must have n_bus + 1 entries");
  gs2g_grid_info g{};
  int rc;
  {
    py::gil_scoped_release nogil;
    rc = gs2g_plan_info(n_bus, indptr.data(), indices.data(), pv.data(), (int)pv.size(), pq.data(), (int)pq.size(),
                        tail_policy, &g);
  }
  check(rc);
  py::dict d;
  d["n_bus"] = g.n_bus;
  d["nnz_y"] = g.nnz_y;
  d["n_pvpq"] = g.n_pvpq;
  d["n_pq"] = g.n_pq;
  d["dim_j"] = g.dim_j;
  d["nnz_j"] = g.nnz_j;
  d["nnz_lu"] = g.nnz_lu;
  d["head_dim"] = g.head_dim;
  d["tail_dim"] = g.tail_dim;
  d["tail_dim_exact"] = g.tail_dim_exact;
  d["n_levels"] = g.n_levels;
  d["n_supernodes"] = g.n_supernodes;
  d["head_madds"] = g.head_madds;
  d["schur_madds"] = g.schur_madds;
  d["dense_madds"] = g.dense_madds;
  d["plan_ms"] = g.plan_ms;
  return d;
}

// Several sessions' current rows in one persistent launch (gs2g_run_multi).
void run_multi(const std::vector<Session*>& sessions, int max_iter, double tol, bool fixed_iters, int precision,
               int start, double pivot_floor, int n_ctas, bool profile, int refactor, double refactor_ratio,
               int max_reuse, bool rescue, int iters_per_round, bool step_scaling, double max_dva,
               double max_dvm) {
  std::vector<gs2g_session*> hs;
  for (Session* s : sessions) {
    if (!s) throw py::value_error("run_multi: None in the session list");
    hs.push_back(reinterpret_cast<gs2g_session*>(s->handle()));
  }
  gs2g_run_opts o = make_opts(max_iter, tol, fixed_iters, precision, start, pivot_floor, n_ctas, profile, refactor,
                              refactor_ratio, max_reuse, rescue, iters_per_round, false, step_scaling, max_dva, max_dvm);
  int rc;
  {
    py::gil_scoped_release nogil;
    rc = gs2g_run_multi(hs.data(), (int)hs.size(), &o);
  }
  check(rc);
}

// ---- warm-start MLP: raw device pointers (integers) from the caller's tensors
template <class T>
T* P(uintptr_t p) {
  return reinterpret_cast<T*>(p);
}
void* S(uintptr_t stream) { return reinterpret_cast<void*>(stream); }

void bind_mlp(py::module_& m) {
  auto mm = m.def_submodule("mlp", "warm-start MLP device routines (include/gs2g.h, gs2g_mlp_*)");
  mm.def("gemm_tn_bf16", [](uintptr_t A, int lda, uintptr_t B, int ldb, uintptr_t D, int ldd, int M, int N, int K,
                            bool accumulate, uintptr_t err, uintptr_t stream) {
    check(gs2g_mlp_gemm_tn_bf16(P<void>(A), lda, P<void>(B), ldb, P<float>(D), ldd, M, N, K, accumulate ? 1 : 0,
                                P<int>(err), S(stream)));
  });
  mm.def("bias_act", [](uintptr_t pre, int ldp, uintptr_t bias, uintptr_t act, int lda, int rows, int cols, bool gelu,
                        uintptr_t stream) {
    check(gs2g_mlp_bias_act(P<float>(pre), ldp, P<float>(bias), P<void>(act), lda, rows, cols, gelu ? 1 : 0,
                            S(stream)));
  });
  mm.def("gelu_bwd", [](uintptr_t dact, int ldg, uintptr_t pre, int ldp, uintptr_t dpre, int ldo, int rows, int cols,
                        uintptr_t stream) {
    check(gs2g_mlp_gelu_bwd(P<float>(dact), ldg, P<float>(pre), ldp, P<void>(dpre), ldo, rows, cols, S(stream)));
  });
  mm.def("mse_grad", [](uintptr_t y, uintptr_t t, int ld, uintptr_t dy, int rows, int cols, int cols_valid,
                        float scale, uintptr_t loss, uintptr_t stream) {
    check(gs2g_mlp_mse_grad(P<float>(y), P<float>(t), ld, P<void>(dy), rows, cols, cols_valid, scale, P<float>(loss),
                            S(stream)));
  });
  mm.def("colsum_bf16", [](uintptr_t x, int ld, int rows, int cols, uintptr_t out, uintptr_t stream) {
    check(gs2g_mlp_colsum_bf16(P<void>(x), ld, rows, cols, P<float>(out), S(stream)));
  });
  mm.def("transpose_bf16", [](uintptr_t in, int ldi, uintptr_t out, int ldo, int rows, int cols, uintptr_t stream) {
    check(gs2g_mlp_transpose_bf16(P<void>(in), ldi, P<void>(out), ldo, rows, cols, S(stream)));
  });
  mm.def("to_bf16", [](uintptr_t in, uintptr_t out, int64_t n, uintptr_t stream) {
    check(gs2g_mlp_to_bf16(P<float>(in), P<void>(out), n, S(stream)));
  });
  mm.def("adam", [](uintptr_t w, uintptr_t g, uintptr_t mo, uintptr_t v, uintptr_t wb, int64_t n, float lr,
                    float b1, float b2, float eps, int step, float wd, uintptr_t stream) {
    check(gs2g_mlp_adam(P<float>(w), P<float>(g), P<float>(mo), P<float>(v), P<void>(wb), n, lr, b1, b2, eps, step,
                        wd, S(stream)));
  });
  mm.def("features", [](uintptr_t sbus_rows, uintptr_t sbus_base, uintptr_t pvpq, int n_pvpq, uintptr_t pq, int n_pq,
                        uintptr_t trip_ptr, uintptr_t trip_ids, uintptr_t br_col, uintptr_t br_val, uintptr_t x_mean,
                        uintptr_t x_std, int n_in, uintptr_t x, int ldx, int rows, int rows_pad, int n_bus,
                        uintptr_t stream) {
    check(gs2g_mlp_features(P<const double>(sbus_rows), P<const double>(sbus_base), P<const int>(pvpq), n_pvpq,
                            P<const int>(pq), n_pq, P<const int>(trip_ptr), P<const int>(trip_ids), P<const int>(br_col),
                            P<const float>(br_val), P<const float>(x_mean), P<const float>(x_std), n_in, P<void>(x),
                            ldx, rows, rows_pad, n_bus, S(stream)));
  });
  mm.def("first_layer_base", [](uintptr_t w0t, int h, uintptr_t x_mean, uintptr_t x_std, int n_in, uintptr_t base,
                                uintptr_t stream) {
    check(gs2g_mlp_first_layer_base(P<const void>(w0t), h, P<const float>(x_mean), P<const float>(x_std), n_in,
                                    P<float>(base), S(stream)));
  });
  mm.def("sparse_first_layer", [](uintptr_t base, uintptr_t w0t, int h, uintptr_t trip_ptr, uintptr_t trip_ids,
                                  uintptr_t br_col, uintptr_t br_val, uintptr_t x_mean, uintptr_t x_std, int n_in,
                                  uintptr_t pre, int ldp, int rows, int rows_pad, uintptr_t stream) {
    check(gs2g_mlp_sparse_first_layer(P<const float>(base), P<const void>(w0t), h, P<const int>(trip_ptr),
                                      P<const int>(trip_ids), P<const int>(br_col), P<const float>(br_val),
                                      P<const float>(x_mean), P<const float>(x_std), n_in, P<float>(pre), ldp, rows,
                                      rows_pad, S(stream)));
  });
  mm.def("start_voltages", [](uintptr_t y, int ldy, uintptr_t ymean, uintptr_t ystd, uintptr_t ia, uintptr_t im,
                              uintptr_t vinit, int n_bus, uintptr_t v0, int rows, uintptr_t stream) {
    check(gs2g_mlp_start_voltages(P<float>(y), ldy, P<float>(ymean), P<float>(ystd), P<int>(ia), P<int>(im),
                                  P<double>(vinit), n_bus, P<double>(v0), rows, S(stream)));
  });
}

}  // namespace

PYBIND11_MODULE(_gs2g, m) {
  m.def("plan_info", &plan_info, py::arg("n_bus"), py::arg("indptr"), py::arg("indices"), py::arg("pv"),
        py::arg("pq"), py::arg("tail_policy") = 1);
  m.doc() = "B200-native batched Newton-Raphson AC power flow (binding of include/gs2g.h)";
  m.attr("PREC_FP64") = GS2G_PREC_FP64;
  m.attr("PREC_MIXED") = GS2G_PREC_MIXED;
  m.attr("START_VINIT") = GS2G_START_VINIT;
  m.attr("START_BASE") = GS2G_START_BASE;
  m.attr("START_ROWS") = GS2G_START_ROWS;
  m.attr("REFACTOR_EVERY") = GS2G_REFACTOR_EVERY;
  m.attr("REFACTOR_ADAPTIVE") = GS2G_REFACTOR_ADAPTIVE;
  m.attr("REFACTOR_BASE_CHORD") = GS2G_REFACTOR_BASE_CHORD;
  m.def("version", &gs2g_version);
  m.def("max_edits_per_row", &gs2g_max_edits_per_row);
  m.def("acpf_nr", &acpf_nr);
  bind_mlp(m);
  m.def("run_multi", &run_multi, py::arg("sessions"), py::arg("max_iter"), py::arg("tol"), py::arg("fixed_iters"),
        py::arg("precision"), py::arg("start"), py::arg("pivot_floor") = 0.0, py::arg("n_ctas") = 0,
        py::arg("profile") = false, py::arg("refactor") = 0, py::arg("refactor_ratio") = 0.0,
        py::arg("max_reuse") = 0, py::arg("rescue") = false, py::arg("iters_per_round") = 1,
        py::arg("step_scaling") = false, py::arg("max_dva") = 0.0, py::arg("max_dvm") = 0.0);
  py::class_<Session>(m, "Session")
      .def(py::init<int, int, IArr, IArr, CArr, CArr, CArr, IArr, IArr, int>(), py::arg("device"), py::arg("n_bus"),
           py::arg("indptr"), py::arg("indices"), py::arg("data"), py::arg("vinit"), py::arg("sbus"), py::arg("pv"),
           py::arg("pq"), py::arg("tail_policy") = 1)
      .def("close", &Session::close)
      .def("handle", &Session::handle)
      .def("info", &Session::info)
      .def("set_branch_data", &Session::set_branch_data)
      .def("set_contingencies", &Session::set_contingencies)
      .def("clear_contingencies", &Session::clear_contingencies)
      .def("set_injections", &Session::set_injections)
      .def("clear_injections", &Session::clear_injections)
      .def("set_start_rows", &Session::set_start_rows)
      .def("set_start_rows_device", &Session::set_start_rows_device)
      .def("start_rows_buffer", &Session::start_rows_buffer)
      .def("set_branch_limits", &Session::set_branch_limits)
      .def("run_subset", &Session::run_subset, py::arg("rows"), py::arg("max_iter"), py::arg("tol"),
           py::arg("fixed_iters"), py::arg("precision"), py::arg("start"), py::arg("pivot_floor") = 0.0,
           py::arg("n_ctas") = 0, py::arg("refactor") = 0, py::arg("refactor_ratio") = 0.0, py::arg("max_reuse") = 0,
           py::arg("rescue") = false, py::arg("iters_per_round") = 1, py::arg("profile") = false,
           py::arg("step_scaling") = false, py::arg("max_dva") = 0.0, py::arg("max_dvm") = 0.0)
      .def("branch_loading", &Session::branch_loading)
      .def("set_chord", &Session::set_chord, py::arg("mode"))
      .def("set_handoff", &Session::set_handoff, py::arg("cluster"))
      .def("set_results_mirror", &Session::set_results_mirror, py::arg("on"))
      .def("set_row_order", &Session::set_row_order, py::arg("on"))
      .def("solve_jt", &Session::solve_jt, py::arg("n_rows"), py::arg("rhs"), py::arg("lam"))
      .def("set_handle_disconnected", &Session::set_handle_disconnected, py::arg("on"))
      .def("replan", &Session::replan, py::arg("tail_policy") = 1, py::arg("dense_rate") = 0.0,
           py::arg("force_tau") = -1)
      .def("set_sbus", &Session::set_sbus)
      .def("set_vinit", &Session::set_vinit)
      .def("solve_base", &Session::solve_base, py::arg("max_iter"), py::arg("tol"), py::arg("precision"),
           py::arg("pivot_floor") = 0.0, py::arg("step_then_check") = true)
      .def("set_base_v", &Session::set_base_v)
      .def("run", &Session::run, py::arg("max_iter"), py::arg("tol"), py::arg("fixed_iters"), py::arg("precision"),
           py::arg("start"), py::arg("pivot_floor") = 0.0, py::arg("n_ctas") = 0, py::arg("profile") = false,
           py::arg("refactor") = 0, py::arg("refactor_ratio") = 0.0, py::arg("max_reuse") = 0,
           py::arg("rescue") = false, py::arg("iters_per_round") = 1, py::arg("step_then_check") = false,
           py::arg("step_scaling") = false, py::arg("max_dva") = 0.0, py::arg("max_dvm") = 0.0)
      .def("factor_counts", &Session::factor_counts)
      .def("n_rows", &Session::n_rows)
      .def("results", &Session::results)
      .def("results_view", [](py::object self) { return self.cast<Session&>().results_view(self); })
      .def("device_results", &Session::device_results)
      .def("dlpack", &Session::dlpack)
      .def("device_rows", &Session::device_rows)
      .def("timings", &Session::timings)
      .def("sync", &Session::sync)
      .def("wait_stream", &Session::wait_stream, py::arg("stream"));
}
