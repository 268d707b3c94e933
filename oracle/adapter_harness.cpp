/*
 * adapter_harness.cpp — CLEO's RunCLEO driving the B200 SDMMethods (TEST INFRASTRUCTURE ONLY).
 *
 * Compiled with CLEO's unmodified sources against the Kokkos-API shim (oracle/Makefile, target
 * `adapter`), and linked with libcleo_b200.so. One call runs CLEO's own timestepping class,
 * RunCLEO (libs/runcleo/runcleo.hpp:72-330: create_supers / create_gbxs from initial conditions,
 * prepare_to_timestep, then start_step / coupldyn_step / sdm_step / proceed_to_next_step until
 * t_end), with one of two SDMMethods:
 *   b200 = 1  the specialisation of include/cleo_b200_sdmmethods.hpp (the domain stepped on the
 *             GPU through the C ABI);
 *   b200 = 0  CLEO's own SDMMethods with Condensation >> collisions and PredCorrMotion, as the
 *             reference build (ref_harness.cpp) composes it.
 * Both runs get the same initial conditions, the same prescribed coupled dynamics (gridbox
 * temperature and vapour changed at every coupling step through CouplingComms::receive_dynamics)
 * and an observer that records the domain superdroplets and the gridbox states at every
 * observation time, which the tests compare.
 */
#include <unistd.h>

#include <atomic>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "../include/cleo_b200.h"
#include "../include/cleo_b200_sdmmethods.hpp"
#include "cartesiandomain/createcartesianmaps.hpp"
#include "ref_plugins.hpp"
#include "runcleo/runcleo.hpp"

namespace {

/* A gridbox-boundaries file in CLEO's binary layout (what cleopy's writebinary writes and
 * initialise/readbinary.cpp:27-103 reads: four u32 [first data byte, global metadata bytes,
 * number of variables, bytes of metadata per variable], the global string, per variable 3 x u32
 * [first byte, bytes per datapoint, datapoints], type and unit characters and an f64 scale
 * factor, then the data): ndims (u64 x 3), gbxidxs (u32), gbxbounds (f64, 6 per gridbox). CLEO's
 * own create_cartesian_maps reads it back, so the maps are built by CLEO's code. */
std::filesystem::path write_gridfile(const cleo_b200_grid* g) {
  static std::atomic<unsigned> serial{0};
  const auto path = std::filesystem::temp_directory_path() /
                    ("cleo_b200_grid_" + std::to_string(getpid()) + "_" +
                     std::to_string(serial++) + ".dat");
  const std::string meta = "gridbox boundaries of an undecomposed Cartesian domain";
  const uint32_t nvars = 3, mbytes = 22, n = g->ngbxs;
  const uint32_t d0 = 16 + (uint32_t)meta.size() + nvars * mbytes;
  std::ofstream f(path, std::ios::binary);
  const auto put = [&](const void* p, size_t bytes) {
    f.write(reinterpret_cast<const char*>(p), (std::streamsize)bytes);
  };
  const uint32_t head[4] = {d0, (uint32_t)meta.size(), nvars, mbytes};
  put(head, sizeof(head));
  put(meta.data(), meta.size());
  const uint32_t b0[3] = {d0, d0 + 24, d0 + 24 + 4 * n};
  const uint32_t bsize[3] = {8, 4, 8}, nvar[3] = {3, n, 6 * n};
  const char vtype[3] = {'Q', 'I', 'd'}, units[3] = {' ', ' ', 'm'};
  const double scale[3] = {1.0, 1.0, 1000.0};
  for (int v = 0; v < 3; ++v) {
    const uint32_t m3[3] = {b0[v], bsize[v], nvar[v]};
    put(m3, sizeof(m3));
    put(&vtype[v], 1);
    put(&units[v], 1);
    put(&scale[v], 8);
  }
  const uint64_t nd[3] = {g->ndims[0], g->ndims[1], g->ndims[2]};
  put(nd, sizeof(nd));
  for (uint32_t i = 0; i < n; ++i) put(&i, 4);
  for (uint32_t i = 0; i < n; ++i) {
    const double b[6] = {g->coord3lo[i], g->coord3hi[i], g->coord1lo[i],
                         g->coord1hi[i], g->coord2lo[i], g->coord2hi[i]};
    put(b, sizeof(b));
  }
  return path;
}

CartesianMaps cleo_maps(const cleo_b200_grid* g, unsigned int nspacedims) {
  const auto path = write_gridfile(g);
  const CartesianMaps maps = create_cartesian_maps(g->ngbxs, nspacedims, path);
  std::filesystem::remove(path);
  return maps;
}

/* one observation: the domain superdroplets and the gridbox states at time t */
struct Record {
  unsigned int t;
  std::vector<Superdrop> supers;
  std::vector<State> states;
};

/* Observer (observers/observers.hpp) recording every `interval` model steps. For CLEO's own
 * SDMMethods it also keys the shim's injected random stream by the SDM step about to run (every
 * run_step covers exactly one SDM step here: the coupling interval is the motion interval). */
struct RecordObserver {
  unsigned int interval;
  std::shared_ptr<std::vector<Record>> out;
  bool key_rng;

  unsigned int next_obs(const unsigned int t) const { return ((t / interval) + 1) * interval; }
  bool on_step(const unsigned int t) const { return t % interval == 0; }
  void before_timestepping(const viewd_constgbx, const subviewd_constsupers) const {}
  void after_timestepping() const {}
  void at_start_step(const unsigned int t, const viewd_constgbx d_gbxs,
                     const subviewd_constsupers d_supers) const {
    if (key_rng) kokkos_shim::set_rng_time(t);
    if (!on_step(t)) return;
    Record r{t, {}, {}};
    const auto hs = Kokkos::create_mirror_view(d_supers);
    Kokkos::deep_copy(hs, d_supers);
    for (size_t k = 0; k < hs.extent(0); ++k) r.supers.push_back(hs(k));
    const auto hg = Kokkos::create_mirror_view(d_gbxs);
    Kokkos::deep_copy(hg, d_gbxs);
    for (size_t ii = 0; ii < hg.extent(0); ++ii) r.states.push_back(hg(ii).state);
    out->push_back(std::move(r));
  }
  SDMMonitor auto get_sdmmonitor() const { return NullSDMMonitor{}; }
};

/* Prescribed coupled dynamics: at coupling step k every gridbox's temperature is the initial one
 * times (1 + amp 1e-3 sin(0.7 k)) and its vapour mixing ratio the initial one times
 * (1 + amp 2e-3 cos(0.3 k)); the other fields keep their values. */
struct PrescribedDynamics {
  unsigned int couplstep;
  std::vector<double> temp0, qvap0;
  double amp;
  unsigned int k = 0;
  void prepare_to_timestep() { k = 0; }
  unsigned int get_couplstep() const { return couplstep; }
  bool on_step(const unsigned int t) const { return t % couplstep == 0; }
  void run_step(const unsigned int t, const unsigned int t_next) {
    if (on_step(t_next)) k = t_next / couplstep;
  }
  double temp(const size_t ii) const { return temp0[ii] * (1.0 + amp * 1e-3 * std::sin(0.7 * k)); }
  double qvap(const size_t ii) const { return qvap0[ii] * (1.0 + amp * 2e-3 * std::cos(0.3 * k)); }
};
struct PrescribedComms {
  template <GridboxMaps GbxMaps, CoupledDynamics CD>
  void send_dynamics(const GbxMaps&, const viewh_gbx, const CD&) const {}
  template <GridboxMaps GbxMaps, CoupledDynamics CD>
  void receive_dynamics(const GbxMaps&, const CD& cd, const viewh_gbx h_gbxs) const {
    for (size_t ii = 0; ii < h_gbxs.extent(0); ++ii) {
      h_gbxs(ii).state.temp = cd.temp(ii);
      h_gbxs(ii).state.qvap = cd.qvap(ii);
    }
  }
};

/* InitialConditions (initialise/initialconditions.hpp:79-94) from arrays */
struct ArraySupers {
  InitSupersData data;
  unsigned int nspacedims;
  size_t get_maxnsupers() const { return data.xis.size(); }
  unsigned int get_nspacedims() const { return nspacedims; }
  InitSupersData fetch_data() const { return data; }
};
struct ArrayGbxs {
  size_t ngbxs;
  std::vector<double> p, t, qv, qc;
  std::vector<std::pair<double, double>> w, u, v;
  size_t get_ngbxs() const { return ngbxs; }
  std::vector<double> press() const { return p; }
  std::vector<double> temp() const { return t; }
  std::vector<double> qvap() const { return qv; }
  std::vector<double> qcond() const { return qc; }
  std::vector<std::pair<double, double>> wvel() const { return w; }
  std::vector<std::pair<double, double>> uvel() const { return u; }
  std::vector<std::pair<double, double>> vvel() const { return v; }
};
struct ArrayInit {
  ArraySupers initsupers;
  ArrayGbxs initgbxs;
};

ArrayInit init_from(const cleo_b200_gbx_state* st, const cleo_b200_supers* sd, size_t n,
                    size_t ngbxs, unsigned int nspacedims) {
  ArrayInit ic{{InitSupersData{}, nspacedims}, ArrayGbxs{ngbxs, {}, {}, {}, {}, {}, {}, {}}};
  InitSupersData& d = ic.initsupers.data;
  d.solutes = {SoluteProperties{}};
  for (size_t k = 0; k < n; ++k) {
    d.sdgbxindexes.push_back(sd->sdgbxindex[k]);
    d.coord3s.push_back(sd->coord3[k]);
    d.coord1s.push_back(sd->coord1[k]);
    d.coord2s.push_back(sd->coord2[k]);
    d.radii.push_back(sd->radius[k]);
    d.msols.push_back(sd->msol[k]);
    d.xis.push_back(sd->xi[k]);
    d.sdIds.push_back(Superdrop::IDType{sd->sdid ? (size_t)sd->sdid[k] : k});
  }
  ArrayGbxs& g = ic.initgbxs;
  for (size_t ii = 0; ii < ngbxs; ++ii) {
    g.p.push_back(st->press[ii]);
    g.t.push_back(st->temp[ii]);
    g.qv.push_back(st->qvap[ii]);
    g.qc.push_back(st->qcond[ii]);
    g.w.push_back({st->wvel_lo[ii], st->wvel_hi[ii]});
    g.u.push_back({st->uvel_lo[ii], st->uvel_hi[ii]});
    g.v.push_back({st->vvel_lo[ii], st->vvel_hi[ii]});
  }
  return ic;
}

template <class SDM>
void run_cleo(const SDM& sdm, PrescribedDynamics& dyn, const ArrayInit& ic, unsigned int t_end) {
  const PrescribedComms comms{};
  const RunCLEO runcleo(sdm, dyn, comms);
  runcleo(ic, t_end);
}

}  // namespace

struct adp_run {
  std::shared_ptr<std::vector<Record>> records = std::make_shared<std::vector<Record>>();
  std::string error;
};

extern "C" {

/* RunCLEO from t = 0 to t_end with couplstep = the motion interval, observing every obsstep, the
 * prescribed dynamics' amplitude amp (0: the states stay the initial ones); b200 selects the
 * SDMMethods. Returns CLEO_OK, or CLEO_ERR_ARGUMENT with the exception's text in adp_error. */
int adp_run_cleo(const cleo_b200_params* p, const cleo_b200_grid* g, const cleo_b200_gbx_state* st,
                 const cleo_b200_supers* sd, size_t nsupers, unsigned int nspacedims,
                 uint32_t t_end, uint32_t obsstep, double amp, int b200, adp_run** out) {
  auto run = std::make_unique<adp_run>();
  *out = nullptr;
  try {
    const unsigned int couplstep = p->motionstep;
    const CartesianMaps maps = cleo_maps(g, nspacedims);
    const ArrayInit ic = init_from(st, sd, nsupers, g->ngbxs, nspacedims);
    std::vector<double> t0(st->temp, st->temp + g->ngbxs), q0(st->qvap, st->qvap + g->ngbxs);
    PrescribedDynamics dyn{couplstep, t0, q0, amp};
    if (b200) {
      const RecordObserver obs{obsstep, run->records, false};
      const auto microphys = b200_microphysics(*p);
      const auto movesupers =
          cartesian_movement(maps, b200_motion<CartesianMaps>(*p), NullBoundaryConditions{});
      const SDMMethods sdm(couplstep, maps, microphys, movesupers, obs);
      run_cleo(sdm, dyn, ic, t_end);
    } else {
      const RecordObserver obs{obsstep, run->records, true};
      const auto movesupers = cartesian_movement(maps, ref_motion(*p), NullBoundaryConditions{});
      const SDMMethods sdm(couplstep, maps, ref_microphysics(*p), movesupers, obs);
      run_cleo(sdm, dyn, ic, t_end);
    }
  } catch (const std::exception& e) {
    run->error = e.what();
    *out = run.release();
    return CLEO_ERR_ARGUMENT;
  }
  *out = run.release();
  return CLEO_OK;
}

const char* adp_error(const adp_run* r) { return r ? r->error.c_str() : ""; }
size_t adp_nobs(const adp_run* r) { return r ? r->records->size() : 0; }

/* observation i: its time, the number of domain superdroplets (written to sd if its arrays hold
 * `cap` entries) and the gridbox states (arrays of ngbxs) */
int adp_obs(const adp_run* r, size_t i, uint32_t* t, size_t* nd, cleo_b200_supers* sd, size_t cap,
            cleo_b200_gbx_state* st) {
  if (!r || i >= r->records->size()) return CLEO_ERR_ARGUMENT;
  const Record& rec = (*r->records)[i];
  *t = rec.t;
  *nd = rec.supers.size();
  if (sd && rec.supers.size() <= cap) {
    for (size_t k = 0; k < rec.supers.size(); ++k) {
      const Superdrop& d = rec.supers[k];
      sd->sdgbxindex[k] = d.get_sdgbxindex();
      sd->coord3[k] = d.get_coord3();
      sd->coord1[k] = d.get_coord1();
      sd->coord2[k] = d.get_coord2();
      sd->xi[k] = d.get_xi();
      sd->radius[k] = d.get_radius();
      sd->msol[k] = d.get_msol();
      if (sd->sdid) sd->sdid[k] = d.sdId.get_value();
    }
  }
  if (st) {
    for (size_t ii = 0; ii < rec.states.size(); ++ii) {
      const State& s = rec.states[ii];
      st->volume[ii] = s.get_volume();
      st->press[ii] = s.press;
      st->temp[ii] = s.temp;
      st->qvap[ii] = s.qvap;
      st->qcond[ii] = s.qcond;
      st->wvel_lo[ii] = s.wvel.first;
      st->wvel_hi[ii] = s.wvel.second;
      st->uvel_lo[ii] = s.uvel.first;
      st->uvel_hi[ii] = s.uvel.second;
      st->vvel_lo[ii] = s.vvel.first;
      st->vvel_hi[ii] = s.vvel.second;
    }
  }
  return sd && rec.supers.size() > cap ? CLEO_ERR_CAPACITY : CLEO_OK;
}

void adp_free(adp_run* r) { delete r; }

}  // extern "C"
