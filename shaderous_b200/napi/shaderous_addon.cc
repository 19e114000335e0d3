// Node N-API addon (node-addon-api) over the C ABI of include/shaderous_b200.h, for the
// reference's TypeScript host: src/sim.ts's Simulation (:465-628) and its callers run() in
// src/ui/api.ts:538 and the headless runner tools/headless/*.mjs.
//
// Not built in this repository: it needs node and the N-API headers (binding.gyp beside this
// file). It binds, one JS class each:
//   Sim      a uniform grid (Sim, src/sim.ts:1938):    step, run, readState, setState,
//            diagnostics, clock, setClock, resetProblem, destroy
//   AmrSim   a block grid (AmrSim, src/amr/amr_sim.ts:178): the same, plus leaves, table,
//            readLeaves, regrid, flags, readBins, binWork
//   Tree     the host block tree (BlockTree, src/amr/tree.ts:106): adapt, refine, table, lists
//   Server   batched serving: submit, drain, cancel, result
// Every failing call throws a JS Error with the library's message, as the reference throws.
// run() blocks the calling thread; a host that keeps its event loop turning wraps it in a
// Napi::AsyncWorker (the library's handles are not re-entrant: one call at a time per handle).
#include <napi.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "shaderous_b200.h"

namespace {

int32_t Int(const Napi::Object& o, const char* k, int32_t dflt) {
  return o.Has(k) ? o.Get(k).ToNumber().Int32Value() : dflt;
}
double Num(const Napi::Object& o, const char* k, double dflt) {
  return o.Has(k) ? o.Get(k).ToNumber().DoubleValue() : dflt;
}

int32_t Recon(const std::string& lim) {
  if (lim == "minmod") return SHZ_RECON_MINMOD;
  if (lim == "mc") return SHZ_RECON_MC;
  if (lim == "vanleer") return SHZ_RECON_VANLEER;
  if (lim == "ppm") return SHZ_RECON_PPM;
  return SHZ_RECON_KOREN;
}

// SimConfig (src/sim.ts:48-265) -> shz_config: n[3] from n and ndim, dx from the problem's box.
shz_config ToConfig(const Napi::Object& o) {
  const int32_t n = Int(o, "n", 64), ndim = Int(o, "ndim", 3);
  const double box = Num(o, "box", 1.0);
  shz_config c;
  shz_config_default(&c, n, ndim >= 2 ? n : 1, ndim == 3 ? n : 1, box / n);
  if (o.Has("eosParams")) c.gamma = Num(o.Get("eosParams").As<Napi::Object>(), "gamma", c.gamma);
  if (o.Has("bcLo") && o.Has("bcHi")) {
    auto lo = o.Get("bcLo").As<Napi::Array>(), hi = o.Get("bcHi").As<Napi::Array>();
    for (uint32_t a = 0; a < 3; a++) {
      c.bc_lo[a] = lo.Get(a).ToNumber().Int32Value();
      c.bc_hi[a] = hi.Get(a).ToNumber().Int32Value();
    }
  }
  c.cfl = Num(o, "cfl", c.cfl);
  c.rho_floor = Num(o, "rhoFloor", c.rho_floor);
  c.p_floor = Num(o, "pFloor", c.p_floor);
  c.eta_dual = Num(o, "etaDual", c.eta_dual);
  c.shock_thresh = Num(o, "shockThresh", c.shock_thresh);
  if (o.Has("limiter")) c.recon = Recon(o.Get("limiter").ToString());
  if (o.Has("riemann")) c.riemann = std::string(o.Get("riemann").ToString()) == "hll" ? SHZ_RIEMANN_HLL : SHZ_RIEMANN_HLLC;
  if (o.Has("isentropicRecon")) c.isentropic = o.Get("isentropicRecon").ToBoolean() ? 1 : 0;
  c.t_end = Num(o, "tEnd", c.t_end);
  c.device = Int(o, "device", 0);
  return c;
}

// { kind: 'sod' | 'kh' | 'tgv' | 'sedov' | 'blast' | ..., a: number[], axis, seed }
shz_problem ToProblem(const Napi::Object& o) {
  static const struct { const char* name; int32_t kind; } KINDS[] = {
      {"sod", SHZ_PROB_SOD}, {"kh", SHZ_PROB_KH}, {"tgv", SHZ_PROB_TGV}, {"sedov", SHZ_PROB_SEDOV},
      {"advect", SHZ_PROB_ADVECT}, {"blast", SHZ_PROB_BLAST}, {"gauss", SHZ_PROB_GAUSS}};
  shz_problem p;
  std::memset(&p, 0, sizeof p);
  const std::string k = o.Get("kind").ToString();
  p.kind = -1;
  for (const auto& e : KINDS)
    if (k == e.name) p.kind = e.kind;
  if (o.Has("a")) {
    auto a = o.Get("a").As<Napi::Array>();
    for (uint32_t i = 0; i < a.Length() && i < 8; i++) p.a[i] = a.Get(i).ToNumber().DoubleValue();
  }
  p.axis = Int(o, "axis", 0);
  p.seed = o.Has("seed") ? (uint64_t)o.Get("seed").ToNumber().Int64Value() : 0;
  return p;
}

shz_run_opts ToRunOpts(Napi::Env env, const Napi::Object& o) {
  shz_run_opts r{o.Has("steps") ? o.Get("steps").ToNumber().Int64Value() : -1,
                 o.Has("until") ? o.Get("until").ToNumber().DoubleValue() : NAN,
                 o.Has("timeoutMs") ? o.Get("timeoutMs").ToNumber().DoubleValue() : 0.0};
  // api.ts:543-544
  if (r.steps < 0 && std::isnan(r.until)) throw Napi::Error::New(env, "run() needs `steps`, `until`, or both");
  return r;
}

// RunResult (src/ui/api.ts:199-210).
Napi::Object FromRunResult(Napi::Env env, const shz_run_result& r) {
  static const char* STOP[] = {"steps", "time", "end", "timeout"};
  auto out = Napi::Object::New(env);
  out.Set("t", r.t);
  out.Set("dt", r.dt);
  out.Set("steps", (double)r.steps);
  out.Set("taken", (double)r.taken);
  out.Set("seconds", r.seconds);
  out.Set("stopped", STOP[r.stopped >= 0 && r.stopped < 4 ? r.stopped : 0]);
  out.Set("lastDt", r.last_dt);
  return out;
}

// Diagnostics (src/sim.ts:1810): float64 totals.
Napi::Object FromDiag(Napi::Env env, const shz_diag& d) {
  auto out = Napi::Object::New(env);
  out.Set("t", d.t);
  out.Set("dt", d.dt);
  out.Set("steps", (double)d.steps);
  out.Set("mass", d.mass);
  auto m = Napi::Array::New(env, 3);
  for (uint32_t i = 0; i < 3; i++) m.Set(i, d.momentum[i]);
  out.Set("momentum", m);
  out.Set("eKin", d.e_kin);
  out.Set("eInt", d.e_int);
  out.Set("eTot", d.e_tot);
  out.Set("maxMach", d.max_mach);
  out.Set("floored", d.floored);
  return out;
}

// ---------------------------------------------------------------------------------------------

class Sim : public Napi::ObjectWrap<Sim> {
 public:
  static Napi::Function Define(Napi::Env env) {
    return DefineClass(env, "Sim",
                       {InstanceMethod("step", &Sim::Step), InstanceMethod("run", &Sim::Run),
                        InstanceMethod("readState", &Sim::ReadState), InstanceMethod("setState", &Sim::SetState),
                        InstanceMethod("resetProblem", &Sim::ResetProblem),
                        InstanceMethod("diagnostics", &Sim::Diagnostics), InstanceMethod("clock", &Sim::Clock),
                        InstanceMethod("setClock", &Sim::SetClock), InstanceMethod("destroy", &Sim::Destroy)});
  }
  explicit Sim(const Napi::CallbackInfo& info) : Napi::ObjectWrap<Sim>(info) {
    shz_config c = ToConfig(info[0].As<Napi::Object>());
    Check(info.Env(), shz_create(&c, &sim_));
    ncell_ = (size_t)c.n[0] * c.n[1] * c.n[2];
  }
  ~Sim() override { shz_destroy(sim_); }

 private:
  void Check(Napi::Env env, int rc) {
    if (rc != SHZ_OK) throw Napi::Error::New(env, sim_ ? shz_last_error(sim_) : shz_last_error(nullptr));
  }
  shz_sim* Live(Napi::Env env) {
    if (!sim_) throw Napi::Error::New(env, "the simulation was destroyed");
    return sim_;
  }
  Napi::Value Step(const Napi::CallbackInfo& info) {
    Check(info.Env(), shz_step(Live(info.Env()), info[0].ToNumber().Int32Value()));
    return info.Env().Undefined();
  }
  Napi::Value Run(const Napi::CallbackInfo& info) {
    shz_run_opts o = ToRunOpts(info.Env(), info[0].As<Napi::Object>());
    shz_run_result r;
    Check(info.Env(), shz_run(Live(info.Env()), &o, &r));
    return FromRunResult(info.Env(), r);
  }
  // readState -> { u1, u2 }: Float32Arrays of 4 ncell, x fastest (src/sim.ts:3790-3808).
  Napi::Value ReadState(const Napi::CallbackInfo& info) {
    auto u1 = Napi::Float32Array::New(info.Env(), 4 * ncell_);
    auto u2 = Napi::Float32Array::New(info.Env(), 4 * ncell_);
    Check(info.Env(), shz_get_state(Live(info.Env()), u1.Data(), u2.Data(), ncell_));
    auto out = Napi::Object::New(info.Env());
    out.Set("u1", u1);
    out.Set("u2", u2);
    return out;
  }
  Napi::Value SetState(const Napi::CallbackInfo& info) {
    auto u1 = info[0].As<Napi::Float32Array>(), u2 = info[1].As<Napi::Float32Array>();
    if (u1.ElementLength() != 4 * ncell_ || u2.ElementLength() != 4 * ncell_)
      throw Napi::RangeError::New(info.Env(), "setState: u1 and u2 must hold 4 floats per cell");
    Check(info.Env(), shz_set_state(Live(info.Env()), u1.Data(), u2.Data(), ncell_));
    return info.Env().Undefined();
  }
  Napi::Value ResetProblem(const Napi::CallbackInfo& info) {
    shz_problem p = ToProblem(info[0].As<Napi::Object>());
    Check(info.Env(), shz_reset_problem(Live(info.Env()), &p));
    return info.Env().Undefined();
  }
  Napi::Value Diagnostics(const Napi::CallbackInfo& info) {
    shz_diag d;
    Check(info.Env(), shz_diagnostics(Live(info.Env()), &d));
    return FromDiag(info.Env(), d);
  }
  Napi::Value Clock(const Napi::CallbackInfo& info) {
    double t = 0, dt = 0;
    int64_t steps = 0;
    Check(info.Env(), shz_clock(Live(info.Env()), &t, &dt, &steps));
    auto out = Napi::Object::New(info.Env());
    out.Set("t", t);
    out.Set("dt", dt);
    out.Set("steps", (double)steps);
    return out;
  }
  Napi::Value SetClock(const Napi::CallbackInfo& info) {
    Check(info.Env(), shz_set_clock(Live(info.Env()), info[0].ToNumber().DoubleValue(), info[1].ToNumber().Int64Value()));
    return info.Env().Undefined();
  }
  Napi::Value Destroy(const Napi::CallbackInfo& info) {
    shz_destroy(sim_);
    sim_ = nullptr;
    return info.Env().Undefined();
  }
  shz_sim* sim_ = nullptr;
  size_t ncell_ = 0;
};

// ---------------------------------------------------------------------------------------------

class AmrSim : public Napi::ObjectWrap<AmrSim> {
 public:
  static Napi::Function Define(Napi::Env env) {
    return DefineClass(
        env, "AmrSim",
        {InstanceMethod("step", &AmrSim::Step), InstanceMethod("run", &AmrSim::Run),
         InstanceMethod("resetProblem", &AmrSim::ResetProblem), InstanceMethod("diagnostics", &AmrSim::Diagnostics),
         InstanceMethod("leaves", &AmrSim::Leaves), InstanceMethod("table", &AmrSim::Table),
         InstanceMethod("readLeaves", &AmrSim::ReadLeaves), InstanceMethod("regrid", &AmrSim::Regrid),
         InstanceMethod("flags", &AmrSim::Flags), InstanceMethod("readBins", &AmrSim::ReadBins),
         InstanceMethod("binWork", &AmrSim::BinWork), InstanceMethod("destroy", &AmrSim::Destroy)});
  }
  // cfg: a SimConfig with amrLevels > 0 (and amrBudget, timeBins, timeBinsAlways), plus the
  // mesh's roots per side (nr) and the refinement thresholds (refineHi, refineLo).
  explicit AmrSim(const Napi::CallbackInfo& info) : Napi::ObjectWrap<AmrSim>(info) {
    auto o = info[0].As<Napi::Object>();
    shz_amr_config c;
    std::memset(&c, 0, sizeof c);
    c.hydro = ToConfig(o);
    c.ndim = Int(o, "ndim", 3);
    c.nr = Int(o, "nr", 2);
    c.max_level = Int(o, "amrLevels", 2);
    c.cap = Int(o, "amrBudget", 4096);
    c.box = Num(o, "box", 1.0);
    c.refine_hi = Num(o, "refineHi", 0.1);
    c.refine_lo = Num(o, "refineLo", 0.05);
    c.regrid_every = Int(o, "regridEvery", 8);  // REGRID_EVERY, amr_sim.ts:73
    c.time_bins = Int(o, "timeBins", 0);
    c.time_bins_always = o.Has("timeBinsAlways") && o.Get("timeBinsAlways").ToBoolean() ? 1 : 0;
    ndim_ = c.ndim;
    cap_ = c.cap;
    Check(info.Env(), shz_amr_create(&c, &a_));
  }
  ~AmrSim() override { shz_amr_destroy(a_); }

 private:
  void Check(Napi::Env env, int rc) {
    if (rc != SHZ_OK) throw Napi::Error::New(env, shz_amr_error(a_));
  }
  shz_amr* Live(Napi::Env env) {
    if (!a_) throw Napi::Error::New(env, "the simulation was destroyed");
    return a_;
  }
  int32_t NLeaves(Napi::Env env) {
    int32_t n = 0;
    std::vector<int32_t> s(cap_), l(cap_), c(3 * (size_t)cap_);
    Check(env, shz_amr_leaves(Live(env), &n, s.data(), l.data(), c.data()));
    return n;
  }
  Napi::Value Step(const Napi::CallbackInfo& info) {
    Check(info.Env(), shz_amr_step(Live(info.Env()), info[0].ToNumber().Int32Value()));
    return info.Env().Undefined();
  }
  Napi::Value Run(const Napi::CallbackInfo& info) {
    shz_run_opts o = ToRunOpts(info.Env(), info[0].As<Napi::Object>());
    shz_run_result r;
    Check(info.Env(), shz_amr_run(Live(info.Env()), &o, &r));
    return FromRunResult(info.Env(), r);
  }
  Napi::Value ResetProblem(const Napi::CallbackInfo& info) {
    shz_problem p = ToProblem(info[0].As<Napi::Object>());
    Check(info.Env(), shz_amr_reset_problem(Live(info.Env()), &p));
    return info.Env().Undefined();
  }
  Napi::Value Diagnostics(const Napi::CallbackInfo& info) {
    shz_diag d;
    Check(info.Env(), shz_amr_diagnostics(Live(info.Env()), &d));
    return FromDiag(info.Env(), d);
  }
  // { slots, levels, coords } of the leaves, coarsest first (BlockTree.lists().leaves).
  Napi::Value Leaves(const Napi::CallbackInfo& info) {
    Napi::Env env = info.Env();
    int32_t n = 0;
    auto s = Napi::Int32Array::New(env, cap_), l = Napi::Int32Array::New(env, cap_), c = Napi::Int32Array::New(env, 3 * cap_);
    Check(env, shz_amr_leaves(Live(env), &n, s.Data(), l.Data(), c.Data()));
    auto out = Napi::Object::New(env);
    out.Set("count", n);
    out.Set("slots", s);
    out.Set("levels", l);
    out.Set("coords", c);
    return out;
  }
  // The block table, cap x 32 ints (BlockTree.table, src/amr/tree.ts:642-679).
  Napi::Value Table(const Napi::CallbackInfo& info) {
    auto t = Napi::Int32Array::New(info.Env(), (size_t)cap_ * 32);
    Check(info.Env(), shz_amr_table(Live(info.Env()), t.Data()));
    return t;
  }
  Napi::Value ReadLeaves(const Napi::CallbackInfo& info) {
    Napi::Env env = info.Env();
    const size_t cells = (size_t)NLeaves(env) * (ndim_ == 3 ? 4096 : 256);
    auto u1 = Napi::Float32Array::New(env, 4 * cells), u2 = Napi::Float32Array::New(env, 4 * cells);
    Check(env, shz_amr_get_leaves_state(Live(env), u1.Data(), u2.Data()));
    auto out = Napi::Object::New(env);
    out.Set("u1", u1);
    out.Set("u2", u2);
    return out;
  }
  Napi::Value Regrid(const Napi::CallbackInfo& info) {
    int32_t changed = 0;
    Check(info.Env(), shz_amr_regrid(Live(info.Env()), &changed));
    return Napi::Boolean::New(info.Env(), changed != 0);
  }
  Napi::Value Flags(const Napi::CallbackInfo& info) {
    auto f = Napi::Float32Array::New(info.Env(), cap_);
    Check(info.Env(), shz_amr_flags(Live(info.Env()), f.Data()));
    return f;
  }
  // AmrSim.readBins (amr_sim.ts:4283): [substep, bin per slot...]
  Napi::Value ReadBins(const Napi::CallbackInfo& info) {
    auto b = Napi::Int32Array::New(info.Env(), (size_t)cap_ + 1);
    Check(info.Env(), shz_amr_bins(Live(info.Env()), b.Data(), nullptr));
    return b;
  }
  // AmrSim.binWork (amr_sim.ts:1663)
  Napi::Value BinWork(const Napi::CallbackInfo& info) {
    int64_t cycles = 0, updates = 0, single = 0;
    int32_t paused = 0;
    Check(info.Env(), shz_amr_bin_work(Live(info.Env()), &cycles, &updates, &single, &paused));
    auto out = Napi::Object::New(info.Env());
    out.Set("cycles", (double)cycles);
    out.Set("updates", (double)updates);
    out.Set("single", (double)single);
    out.Set("paused", paused);
    return out;
  }
  Napi::Value Destroy(const Napi::CallbackInfo& info) {
    shz_amr_destroy(a_);
    a_ = nullptr;
    return info.Env().Undefined();
  }
  shz_amr* a_ = nullptr;
  int ndim_ = 3, cap_ = 0;
};

// ---------------------------------------------------------------------------------------------

class Tree : public Napi::ObjectWrap<Tree> {
 public:
  static Napi::Function Define(Napi::Env env) {
    return DefineClass(env, "Tree",
                       {InstanceMethod("adapt", &Tree::Adapt), InstanceMethod("refine", &Tree::Refine),
                        InstanceMethod("table", &Tree::Table), InstanceMethod("lists", &Tree::Lists)});
  }
  // new Tree(ndim, nr, maxLevel, cap, bcLo, bcHi)
  explicit Tree(const Napi::CallbackInfo& info) : Napi::ObjectWrap<Tree>(info) {
    int32_t lo[3], hi[3];
    auto l = info[4].As<Napi::Array>(), h = info[5].As<Napi::Array>();
    for (uint32_t a = 0; a < 3; a++) {
      lo[a] = l.Get(a).ToNumber().Int32Value();
      hi[a] = h.Get(a).ToNumber().Int32Value();
    }
    cap_ = info[3].ToNumber().Int32Value();
    Check(info.Env(), shz_tree_create(info[0].ToNumber().Int32Value(), info[1].ToNumber().Int32Value(),
                                      info[2].ToNumber().Int32Value(), cap_, lo, hi, 0, &t_));
  }
  ~Tree() override { shz_tree_destroy(t_); }

 private:
  void Check(Napi::Env env, int rc) {
    if (rc != SHZ_OK) throw Napi::Error::New(env, shz_tree_error());
  }
  // adapt(indicatorBySlot: Float64Array, hi, lo) -> regrid table (Int32Array, cap x 12) or null
  Napi::Value Adapt(const Napi::CallbackInfo& info) {
    auto ind = info[0].As<Napi::Float64Array>();
    auto rg = Napi::Int32Array::New(info.Env(), (size_t)cap_ * 12);
    int32_t changed = 0;
    Check(info.Env(), shz_tree_adapt(t_, ind.Data(), info[1].ToNumber().DoubleValue(), info[2].ToNumber().DoubleValue(),
                                     rg.Data(), &changed));
    return changed ? Napi::Value(rg) : info.Env().Null();
  }
  Napi::Value Refine(const Napi::CallbackInfo& info) {
    int32_t c[3];
    auto a = info[1].As<Napi::Array>();
    for (uint32_t i = 0; i < 3; i++) c[i] = a.Get(i).ToNumber().Int32Value();
    int32_t split = 0;
    Check(info.Env(), shz_tree_refine(t_, info[0].ToNumber().Int32Value(), c, &split));
    return Napi::Number::New(info.Env(), split);
  }
  Napi::Value Table(const Napi::CallbackInfo& info) {
    auto t = Napi::Int32Array::New(info.Env(), (size_t)cap_ * 32);
    Check(info.Env(), shz_tree_table(t_, t.Data()));
    return t;
  }
  Napi::Value Lists(const Napi::CallbackInfo& info) {
    Napi::Env env = info.Env();
    std::vector<int32_t> all(cap_), leaves(cap_), per(8);
    int32_t na = 0, nl = 0;
    Check(env, shz_tree_lists(t_, all.data(), leaves.data(), per.data(), &na, &nl));
    auto a = Napi::Uint32Array::New(env, na), l = Napi::Uint32Array::New(env, nl);
    for (int32_t i = 0; i < na; i++) a[i] = (uint32_t)all[i];
    for (int32_t i = 0; i < nl; i++) l[i] = (uint32_t)leaves[i];
    auto out = Napi::Object::New(env);
    out.Set("all", a);
    out.Set("leaves", l);
    return out;
  }
  shz_tree* t_ = nullptr;
  int32_t cap_ = 0;
};

// ---------------------------------------------------------------------------------------------

class Server : public Napi::ObjectWrap<Server> {
 public:
  static Napi::Function Define(Napi::Env env) {
    return DefineClass(env, "Server",
                       {InstanceMethod("submit", &Server::Submit), InstanceMethod("drain", &Server::Drain),
                        InstanceMethod("cancel", &Server::Cancel), InstanceMethod("result", &Server::Result),
                        InstanceMethod("destroy", &Server::Destroy)});
  }
  // new Server({ hydro: SimConfig, budgetBytes, maxGrids, roundSteps })
  explicit Server(const Napi::CallbackInfo& info) : Napi::ObjectWrap<Server>(info) {
    auto o = info[0].As<Napi::Object>();
    shz_server_config c;
    std::memset(&c, 0, sizeof c);
    c.hydro = ToConfig(o.Get("hydro").As<Napi::Object>());
    c.budget_bytes = Num(o, "budgetBytes", 8e9);
    c.max_grids = Int(o, "maxGrids", 256);
    c.round_steps = Int(o, "roundSteps", 8);
    c.keep_states = 0;
    const int rc = shz_server_create(&c, &s_);
    if (rc != SHZ_OK) throw Napi::Error::New(info.Env(), shz_server_error(nullptr));
  }
  ~Server() override { shz_server_destroy(s_); }

 private:
  void Check(Napi::Env env, int rc) {
    if (rc == SHZ_OK) return;
    auto e = Napi::Error::New(env, shz_server_error(s_));
    e.Set("code", Napi::Number::New(env, rc));  // SHZ_E_CANCELLED for a cancelled request
    throw e;
  }
  // submit({ ndim, n, steps, bc, gamma, problem }) -> id
  Napi::Value Submit(const Napi::CallbackInfo& info) {
    auto o = info[0].As<Napi::Object>();
    shz_request r;
    std::memset(&r, 0, sizeof r);
    r.ndim = Int(o, "ndim", 3);
    r.n = Int(o, "n", 64);
    r.steps = Int(o, "steps", 100);
    r.bc = Int(o, "bc", 0);
    r.gamma = Num(o, "gamma", 1.4);
    r.problem = ToProblem(o.Get("problem").As<Napi::Object>());
    int64_t id = 0;
    Check(info.Env(), shz_server_submit(s_, &r, &id));
    return Napi::Number::New(info.Env(), (double)id);
  }
  Napi::Value Drain(const Napi::CallbackInfo& info) {
    Check(info.Env(), shz_server_drain(s_, info.Length() > 0 ? info[0].ToNumber().Int32Value() : 0));
    return info.Env().Undefined();
  }
  Napi::Value Cancel(const Napi::CallbackInfo& info) {
    Check(info.Env(), shz_server_cancel(s_, info[0].ToNumber().Int64Value()));
    return info.Env().Undefined();
  }
  Napi::Value Result(const Napi::CallbackInfo& info) {
    shz_diag d;
    Check(info.Env(), shz_server_result(s_, info[0].ToNumber().Int64Value(), &d));
    return FromDiag(info.Env(), d);
  }
  Napi::Value Destroy(const Napi::CallbackInfo& info) {
    shz_server_destroy(s_);
    s_ = nullptr;
    return info.Env().Undefined();
  }
  shz_server* s_ = nullptr;
};

Napi::Object InitAll(Napi::Env env, Napi::Object exports) {
  exports.Set("Sim", Sim::Define(env));
  exports.Set("AmrSim", AmrSim::Define(env));
  exports.Set("Tree", Tree::Define(env));
  exports.Set("Server", Server::Define(env));
  exports.Set("version", Napi::String::New(env, shz_version()));
  return exports;
}

}  // namespace

NODE_API_MODULE(shaderous_b200, InitAll)
