/*
 * ref_harness.cpp — drives CLEO's own hot-path sources (TEST INFRASTRUCTURE ONLY).
 *
 * Compiled together with the reference's translation units, unmodified, against the
 * project-written Kokkos-API shim in oracle/kokkos_shim (see oracle/Makefile). It builds the
 * reference's own objects — CartesianMaps, Gridbox DualViews, SupersInDomain,
 * MoveSupersInDomain<CartesianMaps, PredCorrMotion, CartesianTransportAcrossDomain,
 * NullBoundaryConditions> and SDMMethods with Condensation >> DoCollisions — and exposes them
 * through the same C-API shape as oracle/cleo_oracle.h (prefix ref_ instead of oc_).
 *
 * The only project code on the arithmetic path is the dispatch below: small structs that satisfy
 * the reference's VelocityFormula / PairProbability / PairEnactX / NFragments / CoalBuReFlag
 * concepts by forwarding to the reference's own implementations, so that one instantiation of
 * SDMMethods serves every plug-in combination selected at run time. DoCollisions is built the
 * way CollCoal/CollBu/CoalBuRe build it (coalescence.hpp:149-160, breakup.hpp:111-123,
 * coalbure.hpp:173-185) and Condensation through its own factory (condensation.hpp:242-253).
 */
#include <cfloat>
#include <filesystem>
#include <cstring>
#include <memory>
#include <string>

#include "../include/cleo_b200.h"
#include "cartesiandomain/cartesianmaps.hpp"
#include "cartesiandomain/movement/cartesian_motion.hpp"
#include "cartesiandomain/movement/cartesian_movement.hpp"
#include "gridboxes/boundary_conditions.hpp"
#include "coupldyn_fromfile/fromfile_cartesian_dynamics.hpp"
#include "initialise/gbx_bounds_from_binary.hpp"
#include "initialise/init_all_supers_from_binary.hpp"
#include "initialise/timesteps.hpp"
#include "observers/collect_data_for_simple_dataset.hpp"
#include "observers/observers.hpp"
#include "observers/sdmmonitor/monitor_massmoments_change.hpp"
#include "observers/superdrops_observer.hpp"
#include "observers/time_observer.hpp"
#include "zarr/fsstore.hpp"
#include "zarr/simple_dataset.hpp"
#include "observers/sdmmonitor/monitor_precipitation_observer.hpp"
#include "runcleo/sdmmethods.hpp"
#include "superdrops/collisions/breakup.hpp"
#include "superdrops/collisions/breakup_nfrags.hpp"
#include "superdrops/collisions/coalbure.hpp"
#include "superdrops/collisions/coalbure_flag.hpp"
#include "superdrops/collisions/coalescence.hpp"
#include "superdrops/collisions/collisions.hpp"
#include "superdrops/collisions/constprob.hpp"
#include "superdrops/collisions/golovinprob.hpp"
#include "superdrops/collisions/longhydroprob.hpp"
#include "superdrops/condensation.hpp"
#include "superdrops/impliciteuler.hpp"
#include "superdrops/microphysicalprocess.hpp"
#include "superdrops/terminalvelocity.hpp"
#include "superdrops/thermodynamic_equations.hpp"
#include "ref_plugins.hpp"

namespace {

/* ---- SDMMonitor: the condensed mass per gridbox (condensation.hpp:149) plus the reference's
 * own MonitorMassMomentsChange (all droplets, raindrops) and MonitorPrecipitation, each active
 * when selected by params.monitors ---- */
using MassMomsMo = MonitorMassMomentsChange<MonitorMassMomentsChangeViews>;
using RainMassMomsMo = MonitorMassMomentsChange<MonitorRainMassMomentsChangeViews>;
struct BudgetMonitor {
  Kokkos::View<double*> cond_mass;
  int mask;
  MassMomsMo mm;
  RainMassMomsMo rmm;
  MonitorPrecipitation pr;
  BudgetMonitor(Kokkos::View<double*> cm, int m, size_t ngbxs)
      : cond_mass(cm), mask(m), mm(ngbxs), rmm(ngbxs), pr(ngbxs) {}
  void reset_monitor() const {
    mm.reset_monitor();
    rmm.reset_monitor();
    pr.reset_monitor();
  }
  KOKKOS_FUNCTION void before_timestepping(const TeamMember& tm,
                                           const subviewd_constsupers s) const {
    if (mask & CLEO_MONITOR_MASSMOMENTS) mm.before_timestepping(tm, s);
    if (mask & CLEO_MONITOR_RAINMASSMOMENTS) rmm.before_timestepping(tm, s);
  }
  KOKKOS_FUNCTION void monitor_condensation(const TeamMember& tm, const double d) const {
    cond_mass(tm.league_rank()) += d;
  }
  KOKKOS_FUNCTION void monitor_microphysics(const TeamMember& tm, const viewd_constsupers s) const {
    if (mask & CLEO_MONITOR_MASSMOMENTS) mm.monitor_microphysics(tm, s);
    if (mask & CLEO_MONITOR_RAINMASSMOMENTS) rmm.monitor_microphysics(tm, s);
  }
  void monitor_motion(const viewd_constgbx d_gbxs, const subviewd_constsupers ds) const {
    if (mask & CLEO_MONITOR_MASSMOMENTS) mm.monitor_motion(d_gbxs, ds);
    if (mask & CLEO_MONITOR_RAINMASSMOMENTS) rmm.monitor_motion(d_gbxs, ds);
  }
  KOKKOS_FUNCTION void monitor_precipitation(const TeamMember& tm, const unsigned int gi,
                                             const auto& maps, Superdrop& d) const {
    if (mask & CLEO_MONITOR_PRECIPITATION) pr.monitor_precipitation(tm, gi, maps, d);
  }
};
struct BudgetObserver {
  BudgetMonitor mo;
  void before_timestepping(const viewd_constgbx, const subviewd_constsupers) const {}
  void after_timestepping() const {}
  unsigned int next_obs(const unsigned int) const { return LIMITVALUES::uintmax; }
  bool on_step(const unsigned int) const { return false; }
  void at_start_step(const unsigned int, const viewd_constgbx, const subviewd_constsupers) const {}
  SDMMonitor auto get_sdmmonitor() const { return mo; }
};

using MoveT = MoveSupersInDomain<CartesianMaps, MotionT, CartesianTransportAcrossDomain,
                                 NullBoundaryConditions>;
using SDM = SDMMethods<CartesianMaps, Microphys, MotionT, CartesianTransportAcrossDomain,
                       NullBoundaryConditions, BudgetObserver>;

int code_of(const std::string& m) {
  if (m.find("xi should not be less than 1") != std::string::npos) return CLEO_ERR_XI_ZERO;
  if (m.find("less than dry radius") != std::string::npos) return CLEO_ERR_RADIUS_BELOW_DRY;
  if (m.find("condensate mass cannot") != std::string::npos) return CLEO_ERR_NEG_CONDENSATE;
  if (m.find("coalescence") != std::string::npos || m.find("colllision") != std::string::npos)
    return CLEO_ERR_COALESCENCE;
  if (m.find("nfrags") != std::string::npos) return CLEO_ERR_BREAKUP;
  if (m.find("No root converged") != std::string::npos) return CLEO_ERR_NR_NOCONVERGE;
  if (m.find("subtimestep") != std::string::npos) return CLEO_ERR_SUBDELT;
  if (m.find("CFL") != std::string::npos) return CLEO_ERR_CFL;
  if (m.find("SD not in previous gbx") != std::string::npos) return CLEO_ERR_OUT_OF_BOX;
  if (m.find("psat ERROR") != std::string::npos) return CLEO_ERR_TEMPERATURE;
  return CLEO_ERR_ARGUMENT;
}

}  // namespace

struct ref_ctx {
  cleo_b200_params p;
  uint32_t ngbxs;
  CartesianMaps gbxmaps;
  std::unique_ptr<SDM> sdm;
  dualview_gbx gbxs;
  std::unique_ptr<SupersInDomain> allsupers;
  Kokkos::View<double*> cond_mass;
  std::unique_ptr<BudgetMonitor> mon;
  cleo_b200_error err{CLEO_OK, 0xFFFFFFFFu, 0};
};

/* ---- superdroplet output: the reference's own SimpleDataset<FSStore> with TimeObserver >>
 * SuperdropsObserver collecting all eight variables, composed as the examples compose them
 * (main_rshaft1d.cpp:111-123, main_rshaft1d.cpp:134) ---- */
using ZDataset = SimpleDataset<FSStore>;
struct ZarrObsBase {
  virtual ~ZarrObsBase() = default;
  virtual void at_start_step(unsigned int t, const viewd_constgbx g,
                             const subviewd_constsupers s) const = 0;
};
template <class O>
struct ZarrObs final : ZarrObsBase {
  O obs;
  explicit ZarrObs(O o) : obs(std::move(o)) {}
  void at_start_step(unsigned int t, const viewd_constgbx g,
                     const subviewd_constsupers s) const override {
    if (obs.on_step(t)) obs.at_start_step(t, g, s);
  }
};
template <class O>
static std::unique_ptr<ZarrObsBase> make_zarr_obs(O o) {
  return std::make_unique<ZarrObs<O>>(std::move(o));
}
struct ref_zarr {
  FSStore store;
  ZDataset dataset;
  std::unique_ptr<ZarrObsBase> obs;
  viewd_gbx nogbxs;
  ref_zarr(const char* dir, size_t maxchunk, unsigned int interval)
      : store(std::filesystem::path(dir)), dataset(store), nogbxs("nogbxs", 0) {
    const Observer auto t = TimeObserver(interval, dataset, store, maxchunk, &step2dimlesstime);
    const auto sdid = CollectSdId(dataset, maxchunk);
    const auto sdgbxindex = CollectSdgbxindex(dataset, maxchunk);
    const auto xi = CollectXi(dataset, maxchunk);
    const auto radius = CollectRadius(dataset, maxchunk);
    const auto msol = CollectMsol(dataset, maxchunk);
    const auto coord3 = CollectCoord3(dataset, maxchunk);
    const auto coord1 = CollectCoord1(dataset, maxchunk);
    const auto coord2 = CollectCoord2(dataset, maxchunk);
    const auto all = coord3 >> coord1 >> coord2 >> msol >> radius >> xi >> sdgbxindex >> sdid;
    const Observer auto sd = SuperdropsObserver(interval, dataset, store, maxchunk, all);
    obs = make_zarr_obs(t >> sd);
  }
  ~ref_zarr() { obs.reset(); }  // the observers write their last chunks and shapes here
};

static viewd_supers supers_from_soa(const cleo_b200_supers* h, size_t n) {
  viewd_supers totsupers("totsupers", n);
  for (size_t k = 0; k < n; ++k) {
    const SuperdropAttrs attrs(SoluteProperties{}, h->xi[k], h->radius[k], h->msol[k], true);
    totsupers(k) = Superdrop(h->sdgbxindex[k], h->coord3[k], h->coord1[k], h->coord2[k], attrs,
                             IntID{h->sdid ? (size_t)h->sdid[k] : k});
  }
  return totsupers;
}

static void fail(ref_ctx* c, int code) {
  if (c->err.code == CLEO_OK) c->err.code = code;
}

extern "C" {

void ref_set_num_threads(int n) { kokkos_shim::set_num_threads(n); }

int ref_create(const cleo_b200_params* p, const cleo_b200_grid* g, size_t capacity,
               ref_ctx** out) {
  if (!p || !g || !out) return CLEO_ERR_ARGUMENT;
  auto c = std::make_unique<ref_ctx>();
  c->p = *p;
  c->ngbxs = g->ngbxs;
  try {
    c->gbxmaps = ref_cartesian_maps(g, nullptr);
    const auto P = c->p;
    const Microphys microphys = ref_microphysics(P);
    const MoveT movesupers = cartesian_movement(c->gbxmaps, ref_motion(P), NullBoundaryConditions{});

    c->cond_mass = Kokkos::View<double*>("cond_mass", g->ngbxs);
    c->mon = std::make_unique<BudgetMonitor>(c->cond_mass, P.monitors, g->ngbxs);
    BudgetObserver obs{*c->mon};
    const unsigned int couplstep = P.motionstep == CLEO_STEP_OFF ? 1u : P.motionstep;
    c->sdm = std::make_unique<SDM>(couplstep, c->gbxmaps, microphys, movesupers, obs);
    c->gbxs = dualview_gbx("gbxs", g->ngbxs);
    (void)capacity;
  } catch (const kokkos_shim::Abort& e) {
    return code_of(e.what());
  }
  *out = c.release();
  return CLEO_OK;
}

void ref_destroy(ref_ctx* c) { delete c; }

int ref_upload_supers(ref_ctx* c, const cleo_b200_supers* h, size_t n) {
  try {
    viewd_supers totsupers = supers_from_soa(h, n);
    c->allsupers = std::make_unique<SupersInDomain>(totsupers, c->ngbxs);
    /* gridboxes refer to the sorted superdroplets (Gridbox ctor, gridbox.hpp:44-46) */
    auto hg = c->gbxs.view_host();
    for (unsigned int ii = 0; ii < c->ngbxs; ++ii) {
      const State st = hg(ii).state;
      hg(ii) = Gridbox(Gbxindex{ii}, st, c->allsupers->domain_supers_readonly());
    }
  } catch (const kokkos_shim::Abort& e) {
    fail(c, code_of(e.what()));
    return c->err.code;
  }
  return CLEO_OK;
}

int ref_upload_state(ref_ctx* c, const cleo_b200_gbx_state* h) {
  auto hg = c->gbxs.view_host();
  for (unsigned int ii = 0; ii < c->ngbxs; ++ii) {
    const State st(h->volume[ii], h->press[ii], h->temp[ii], h->qvap[ii], h->qcond[ii],
                   {h->wvel_lo[ii], h->wvel_hi[ii]}, {h->uvel_lo[ii], h->uvel_hi[ii]},
                   {h->vvel_lo[ii], h->vvel_hi[ii]});
    if (c->allsupers) {
      hg(ii) = Gridbox(Gbxindex{ii}, st, c->allsupers->domain_supers_readonly());
    } else {
      hg(ii).gbxindex = Gbxindex{ii};
      hg(ii).state = st;
    }
  }
  return CLEO_OK;
}

/* One SDMMethods::run_step call per SDM step, so that the injected stream is keyed by t_sdm. */
int ref_step(ref_ctx* c, uint32_t t_mdl, uint32_t t_next) {
  if (c->err.code != CLEO_OK) return c->err.code;
  try {
    uint32_t t_sdm = t_mdl;
    while (t_sdm < t_next) {
      uint32_t next_move = CLEO_STEP_OFF;
      if (c->p.motionstep != CLEO_STEP_OFF) next_move = ((t_sdm / c->p.motionstep) + 1) * c->p.motionstep;
      const uint32_t t_sdm_next = t_next < next_move ? t_next : next_move;
      kokkos_shim::set_rng_time(t_sdm);
      c->sdm->run_step(t_sdm, t_sdm_next, c->gbxs.view_device(), *c->allsupers);
      t_sdm = t_sdm_next;
    }
  } catch (const kokkos_shim::Abort& e) {
    fail(c, code_of(e.what()));
  }
  return c->err.code;
}

int ref_status(ref_ctx* c, cleo_b200_error* err) {
  if (err) *err = c->err;
  return c->err.code;
}

int ref_download_supers(ref_ctx* c, cleo_b200_supers* h, size_t* n_domain, size_t* n_total) {
  const auto tot = c->allsupers->get_totsupers_readonly();
  for (size_t k = 0; k < tot.extent(0); ++k) {
    const Superdrop& d = tot(k);
    h->sdgbxindex[k] = d.get_sdgbxindex();
    h->coord3[k] = d.get_coord3();
    h->coord1[k] = d.get_coord1();
    h->coord2[k] = d.get_coord2();
    h->xi[k] = d.get_xi();
    h->radius[k] = d.get_radius();
    h->msol[k] = d.get_msol();
    if (h->sdid) h->sdid[k] = d.sdId.get_value();
  }
  if (n_domain) *n_domain = c->allsupers->domain_nsupers();
  if (n_total) *n_total = tot.extent(0);
  return CLEO_OK;
}

int ref_download_state(ref_ctx* c, cleo_b200_gbx_state* h) {
  const auto hg = c->gbxs.view_host();
  for (unsigned int ii = 0; ii < c->ngbxs; ++ii) {
    const State& s = hg(ii).state;
    h->volume[ii] = s.get_volume();
    h->press[ii] = s.press;
    h->temp[ii] = s.temp;
    h->qvap[ii] = s.qvap;
    h->qcond[ii] = s.qcond;
    h->wvel_lo[ii] = s.wvel.first; h->wvel_hi[ii] = s.wvel.second;
    h->uvel_lo[ii] = s.uvel.first; h->uvel_hi[ii] = s.uvel.second;
    h->vvel_lo[ii] = s.vvel.first; h->vvel_hi[ii] = s.vvel.second;
  }
  return CLEO_OK;
}

/* before_timestepping of the monitors over every gridbox (as DoSDMMonitorObs does,
 * do_sdmmonitor_obs.hpp) and reset_monitor */
int ref_monitors_begin(ref_ctx* c) {
  try {
    const auto d_gbxs = c->gbxs.view_device();
    const auto domainsupers = c->allsupers->domain_supers_readonly();
    const BudgetMonitor mon = *c->mon;
    Kokkos::parallel_for(
        "monitors_begin", TeamPolicy(c->ngbxs, Kokkos::AUTO()),
        [=](const TeamMember& tm) {
          const auto ii = tm.league_rank();
          mon.before_timestepping(tm, d_gbxs(ii).supersingbx.readonly(domainsupers));
        });
    mon.reset_monitor();
  } catch (const kokkos_shim::Abort& e) {
    return code_of(e.what());
  }
  return CLEO_OK;
}

int ref_download_monitors(ref_ctx* c, cleo_b200_monitors* o, int reset) {
  const BudgetMonitor& m = *c->mon;
  for (unsigned int ii = 0; ii < c->ngbxs; ++ii) {
    if (o->mom0_micro) o->mom0_micro[ii] = m.mm.microphysics_moms.d_delta_mom0(ii);
    if (o->mom1_micro) o->mom1_micro[ii] = m.mm.microphysics_moms.d_delta_mom1(ii);
    if (o->mom2_micro) o->mom2_micro[ii] = m.mm.microphysics_moms.d_delta_mom2(ii);
    if (o->mom0_motion) o->mom0_motion[ii] = m.mm.motion_moms.d_delta_mom0(ii);
    if (o->mom1_motion) o->mom1_motion[ii] = m.mm.motion_moms.d_delta_mom1(ii);
    if (o->mom2_motion) o->mom2_motion[ii] = m.mm.motion_moms.d_delta_mom2(ii);
    if (o->rain_mom0_micro) o->rain_mom0_micro[ii] = m.rmm.microphysics_moms.d_delta_mom0(ii);
    if (o->rain_mom1_micro) o->rain_mom1_micro[ii] = m.rmm.microphysics_moms.d_delta_mom1(ii);
    if (o->rain_mom2_micro) o->rain_mom2_micro[ii] = m.rmm.microphysics_moms.d_delta_mom2(ii);
    if (o->rain_mom0_motion) o->rain_mom0_motion[ii] = m.rmm.motion_moms.d_delta_mom0(ii);
    if (o->rain_mom1_motion) o->rain_mom1_motion[ii] = m.rmm.motion_moms.d_delta_mom1(ii);
    if (o->rain_mom2_motion) o->rain_mom2_motion[ii] = m.rmm.motion_moms.d_delta_mom2(ii);
    if (o->precip) o->precip[ii] = m.pr.d_data(ii);
  }
  if (reset) m.reset_monitor();
  return CLEO_OK;
}

/* ---- CLEO's binary initialisation and coupled-dynamics readers ---- */
/* GbxBoundsFromBinary (gbx_bounds_from_binary.cpp): bounds [6 per gridbox], area, volume */
int ref_read_gridfile(const char* path, size_t ngbxs, unsigned int nspacedims, double* bounds,
                      double* areas, double* vols) {
  try {
    const GbxBoundsFromBinary gfb(ngbxs, nspacedims, std::filesystem::path(path));
    for (unsigned int i = 0; i < ngbxs; ++i) {
      const auto b3 = gfb.get_coord3gbxbounds(i), b1 = gfb.get_coord1gbxbounds(i),
                 b2 = gfb.get_coord2gbxbounds(i);
      const double b[6] = {b3.first, b3.second, b1.first, b1.second, b2.first, b2.second};
      for (int k = 0; k < 6; ++k) bounds[6 * i + k] = b[k];
      areas[i] = gfb.gbxarea(i);
      vols[i] = gfb.gbxvol(i);
    }
  } catch (const std::exception&) {
    return CLEO_ERR_ARGUMENT;
  }
  return CLEO_OK;
}

/* InitAllSupersFromBinary (init_all_supers_from_binary.cpp) */
int ref_read_initsupers(const char* path, size_t maxnsupers, unsigned int nspacedims,
                        uint32_t* gbx, uint64_t* xi, double* radius, double* msol, double* c3,
                        double* c1, double* c2) {
  try {
    const InitAllSupersFromBinary init(maxnsupers, std::filesystem::path(path), nspacedims);
    const InitSupersData d = init.fetch_data();
    for (size_t k = 0; k < maxnsupers; ++k) {
      gbx[k] = d.sdgbxindexes.at(k);
      xi[k] = d.xis.at(k);
      radius[k] = d.radii.at(k);
      msol[k] = d.msols.at(k);
      c3[k] = k < d.coord3s.size() ? d.coord3s[k] : 0.0;
      c1[k] = k < d.coord1s.size() ? d.coord1s[k] : 0.0;
      c2[k] = k < d.coord2s.size() ? d.coord2s[k] : 0.0;
    }
  } catch (const std::exception&) {
    return CLEO_ERR_ARGUMENT;
  }
  return CLEO_OK;
}

/* CartesianDynamics (fromfile_cartesian_dynamics.cpp) after `step` increments, read the way
 * FromFileComms::update_gridbox_state does (fromfilecomms.cpp:40-52). paths: press, temp,
 * qvap, qcond, wvel, uvel, vvel. out: press, temp, qvap, qcond, wlo, whi, ulo, uhi, vlo, vhi. */
int ref_fromfile_state(const char* const* paths, unsigned int nspacedims, const uint64_t* ndims,
                       unsigned int nsteps, unsigned int step, double* const* out) {
  try {
    OptionalConfigParams::FromFileDynamicsParams cfg;
    cfg.nspacedims = nspacedims;
    cfg.press = paths[0];
    cfg.temp = paths[1];
    cfg.qvap = paths[2];
    cfg.qcond = paths[3];
    cfg.wvel = paths[4];
    cfg.uvel = paths[5];
    cfg.vvel = paths[6];
    CartesianDynamics dyn(cfg, {ndims[0], ndims[1], ndims[2]}, nsteps);
    for (unsigned int s = 0; s < step; ++s) dyn.increment_position();
    const size_t ng = ndims[0] * ndims[1] * ndims[2];
    for (size_t ii = 0; ii < ng; ++ii) {
      out[0][ii] = dyn.get_press(ii);
      out[1][ii] = dyn.get_temp(ii);
      out[2][ii] = dyn.get_qvap(ii);
      out[3][ii] = dyn.get_qcond(ii);
      const auto w = dyn.get_wvel(ii), u = dyn.get_uvel(ii), v = dyn.get_vvel(ii);
      out[4][ii] = w.first; out[5][ii] = w.second;
      out[6][ii] = u.first; out[7][ii] = u.second;
      out[8][ii] = v.first; out[9][ii] = v.second;
    }
  } catch (const std::exception&) {
    return CLEO_ERR_ARGUMENT;
  }
  return CLEO_OK;
}

int ref_download_budgets(ref_ctx* c, double* cond_mass, uint64_t* nr_iters) {
  for (unsigned int ii = 0; ii < c->ngbxs; ++ii) {
    if (cond_mass) cond_mass[ii] = c->cond_mass(ii);
    if (nr_iters) nr_iters[ii] = 0; /* not observable in the reference */
  }
  return CLEO_OK;
}

/* ImplicitEuler::solve_condensation for independent droplets, set up like
 * DoCondensation::superdroplets_change / superdrop_mass_change (condensation.cpp:43-112). */
int ref_condensation_solve(const cleo_b200_params* p, size_t n, const double* radius,
                           const double* msol, const double* temp, const double* press,
                           const double* s_ratio, const double* delt, double* radius_out) {
  int code = CLEO_OK;
  for (size_t i = 0; i < n; ++i) {
    try {
      const ImplicitEuler impe(delt[i], p->maxniters, p->rtol, p->atol, p->cond_minsubdelt);
      Superdrop drop(0u, 0.0, 0.0, 0.0,
                     SuperdropAttrs(SoluteProperties{}, 1, radius[i], msol[i], true), IntID{i});
      const auto psat = saturation_pressure(temp[i]);
      const auto ffactor = diffusion_factor(press[i], temp[i], psat);
      const auto ab = kohler_factors(drop, temp[i]);
      const auto newr = impe.solve_condensation(s_ratio[i], ab, ffactor, drop.get_radius());
      drop.change_radius(newr);
      radius_out[i] = drop.get_radius();
    } catch (const kokkos_shim::Abort& e) {
      if (code == CLEO_OK) code = code_of(e.what());
      radius_out[i] = NAN;
    }
  }
  return code;
}

double ref_terminal_velocity(int kind, double radius) {
  const Superdrop d(0u, 0.0, 0.0, 0.0, SuperdropAttrs(SoluteProperties{}, 1, radius, 0.0, true),
                    IntID{0});
  return AnyTV{kind}(d);
}

double ref_pair_probability(const cleo_b200_params* p, double r1, uint64_t xi1, double msol1,
                            double r2, uint64_t xi2, double msol2, double volume) {
  const Superdrop a(0u, 0.0, 0.0, 0.0, SuperdropAttrs(SoluteProperties{}, xi1, r1, msol1, true),
                    IntID{0});
  const Superdrop b(0u, 0.0, 0.0, 0.0, SuperdropAttrs(SoluteProperties{}, xi2, r2, msol2, true),
                    IntID{1});
  const AnyProb prob(p->coll_prob, p->coaleff, p->const_kernel);
  return prob(a, b, p->coll_delt, volume * dlc::VOL0);
}

/* Neighbour maps as the reference builds them (doubly_periodic_domain.hpp:41-101 via
 * createcartesianmaps.cpp:203-220) for a 3-D domain; used to pin the host-side grid builder. */
/* Superdroplet output through the reference's writer into directory `dir`: observations every
 * `interval` model steps, arrays chunked by `maxchunk` elements. */
int ref_zarr_open(const char* dir, size_t maxchunk, uint32_t interval, ref_zarr** out) {
  if (!dir || !out || maxchunk == 0 || interval == 0) return CLEO_ERR_ARGUMENT;
  try {
    *out = new ref_zarr(dir, maxchunk, interval);
  } catch (const std::exception&) {
    return CLEO_ERR_ARGUMENT;
  }
  return CLEO_OK;
}

/* SDMMethods::at_start_step (sdmmethods.hpp:300-305): observe the domain superdroplets */
int ref_zarr_observe(ref_zarr* z, ref_ctx* c, uint32_t t_mdl) {
  if (!z || !c || !c->allsupers) return CLEO_ERR_ARGUMENT;
  try {
    z->obs->at_start_step(t_mdl, c->gbxs.view_device(), c->allsupers->domain_supers_readonly());
  } catch (const kokkos_shim::Abort& e) {
    return CLEO_ERR_ARGUMENT;
  }
  return CLEO_OK;
}

/* the same observation of n given superdroplets (taken as the domain superdroplets) */
int ref_zarr_observe_supers(ref_zarr* z, uint32_t t_mdl, const cleo_b200_supers* h, size_t n) {
  if (!z || (!h && n)) return CLEO_ERR_ARGUMENT;
  try {
    const viewd_supers v = supers_from_soa(h, n);
    const subviewd_constsupers s = Kokkos::subview(viewd_constsupers(v), kkpair_size_t({0, n}));
    z->obs->at_start_step(t_mdl, z->nogbxs, s);
  } catch (const kokkos_shim::Abort& e) {
    return CLEO_ERR_ARGUMENT;
  }
  return CLEO_OK;
}

void ref_zarr_close(ref_zarr* z) { delete z; }

void ref_cartesian_neighbours(const uint32_t ndims[3], uint32_t idx, uint32_t out[6]) {
  const std::vector<size_t> nd{ndims[0], ndims[1], ndims[2]};
  const auto z = DoublyPeriodicDomain::cartesian_coord3nghbrs(idx, nd);
  const auto x = DoublyPeriodicDomain::cartesian_coord1nghbrs(idx, nd);
  const auto y = DoublyPeriodicDomain::cartesian_coord2nghbrs(idx, nd);
  out[0] = z.first; out[1] = z.second; out[2] = x.first;
  out[3] = x.second; out[4] = y.first; out[5] = y.second;
}

}  // extern "C"
