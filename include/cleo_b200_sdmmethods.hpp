/*
 * cleo_b200_sdmmethods.hpp — CLEO's SDMMethods on the B200 path (C++ adapter over cleo_b200.h).
 *
 * For a host program built with CLEO's headers (CLEO's libs/ directory on the include path) that
 * runs RunCLEO. CLEO's microphysics and motion plug-ins are evaluated per gridbox inside a Kokkos
 * team (MicrophysicalProcess::run_step, libs/superdrops/microphysicalprocess.hpp:45-52, called in
 * libs/runcleo/sdmmethods.hpp:70-92), and a whole-domain GPU step cannot be started from there.
 * So this header specialises SDMMethods itself (libs/runcleo/sdmmethods.hpp:110-333) for two
 * parameter-carrying plug-in types, B200Microphysics and B200Motion, which still satisfy CLEO's
 * concepts. The specialisation has the primary template's public interface — the constructor,
 * prepare_to_timestep, at_start_step, run_step, get_couplstep, next_couplstep and the members
 * gbxmaps, obs, microphys — so RunCLEO (libs/runcleo/runcleo.hpp:72,277) and a main that builds
 * its SDMMethods with the factories below compile unchanged and step the domain through
 * libcleo_b200.so:
 *
 *   const auto p = ...;                                 // cleo_b200_params: the factory arguments
 *   const auto microphys = b200_microphysics(p);        // in place of Condensation >> collisions
 *   const auto motion = b200_motion<CartesianMaps>(p);  // in place of CartesianMotion(...)
 *   const auto movesupers = cartesian_movement(gbxmaps, motion, NullBoundaryConditions{});
 *   const SDMMethods sdm(couplstep, gbxmaps, microphys, movesupers, obs);
 *   RunCLEO(sdm, coupldyn, comms)(initconds, t_end);
 *
 * Data flow (the device context owns the superdroplets and gridbox states in SoA form):
 *   prepare_to_timestep  creates the context from the parameters and CartesianMaps (bounds,
 *                        neighbours, areas copied out of the maps), uploads the gridbox states
 *                        and all superdroplets, then calls obs.before_timestepping;
 *   run_step             uploads the gridbox states at coupling times (coupled dynamics writes
 *                        them between steps), steps the context (cleo_b200_step), throws
 *                        std::runtime_error on a recorded failure (where CLEO aborts), and
 *                        before a coupling or observation time copies the states back into the
 *                        Gridboxes; before an observation time it also copies the superdroplets
 *                        back into SupersInDomain (SoA to CLEO's AoS) and resets the gridboxes'
 *                        references, so observers see CLEO's data structures as CLEO leaves them;
 *   at_start_step        calls obs.at_start_step, as the primary template does.
 * The observer's SDMMonitor is not called: the B200 step keeps its own budgets and monitors
 * (cleo_b200_download_budgets, cleo_b200_download_monitors).
 */
#ifndef CLEO_B200_SDMMETHODS_HPP_
#define CLEO_B200_SDMMETHODS_HPP_

#include <Kokkos_Core.hpp>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cartesiandomain/cartesianmaps.hpp"
#include "cartesiandomain/movement/cartesian_transport_across_domain.hpp"
#include "cleo_b200.h"
#include "gridboxes/boundary_conditions.hpp"
#include "gridboxes/movesupersindomain.hpp"
#include "runcleo/sdmmethods.hpp"
#include "superdrops/microphysicalprocess.hpp"
#include "superdrops/motion.hpp"

namespace cleo_b200_adapter {

/* next time on an interval's grid, or never for a switched-off process
 * (ConstTstepMicrophysics::next_step, microphysicalprocess.hpp) */
KOKKOS_INLINE_FUNCTION unsigned int next_on(const unsigned int interval, const unsigned int t) {
  return interval == CLEO_STEP_OFF ? LIMITVALUES::uintmax : ((t / interval) + 1) * interval;
}
KOKKOS_INLINE_FUNCTION bool on(const unsigned int interval, const unsigned int t) {
  return interval != CLEO_STEP_OFF && t % interval == 0;
}

[[noreturn]] inline void fail(const int code, const char* where) {
  throw std::runtime_error(std::string("cleo_b200: ") + where + " reported status " +
                           std::to_string(code));
}
inline void check(const int code, const char* where) {
  if (code != CLEO_OK) fail(code, where);
}

/* The device context and the host staging of the exchanges; shared by the copies of one
 * SDMMethods (its methods are const, as the primary template's are). */
struct Device {
  cleo_b200_ctx* ctx = nullptr;
  size_t ngbxs = 0, nsupers = 0;
  std::vector<double> st[11];
  Device() = default;
  Device(const Device&) = delete;
  Device& operator=(const Device&) = delete;
  ~Device() { cleo_b200_destroy(ctx); }
  cleo_b200_gbx_state state_arrays() {
    double* s[11];
    for (int k = 0; k < 11; ++k) {
      st[k].resize(ngbxs ? ngbxs : 1);
      s[k] = st[k].data();
    }
    return cleo_b200_gbx_state{s[0], s[1], s[2], s[3], s[4], s[5],
                               s[6], s[7], s[8], s[9], s[10]};
  }
};

/* the gridboxes' states <-> the context (11 fields per gridbox, State of state.hpp:33-120) */
inline void upload_states(Device& dev, const viewd_constgbx d_gbxs) {
  const auto h = Kokkos::create_mirror_view(d_gbxs);
  Kokkos::deep_copy(h, d_gbxs);
  cleo_b200_gbx_state a = dev.state_arrays();
  for (size_t ii = 0; ii < dev.ngbxs; ++ii) {
    const State& s = h(ii).state;
    a.volume[ii] = s.get_volume();
    a.press[ii] = s.press;
    a.temp[ii] = s.temp;
    a.qvap[ii] = s.qvap;
    a.qcond[ii] = s.qcond;
    a.wvel_lo[ii] = s.wvel.first;
    a.wvel_hi[ii] = s.wvel.second;
    a.uvel_lo[ii] = s.uvel.first;
    a.uvel_hi[ii] = s.uvel.second;
    a.vvel_lo[ii] = s.vvel.first;
    a.vvel_hi[ii] = s.vvel.second;
  }
  check(cleo_b200_upload_state(dev.ctx, &a), "cleo_b200_upload_state");
}
inline void download_states(Device& dev, const viewd_gbx d_gbxs) {
  cleo_b200_gbx_state a = dev.state_arrays();
  check(cleo_b200_download_state(dev.ctx, &a), "cleo_b200_download_state");
  const auto h = Kokkos::create_mirror_view(d_gbxs);
  Kokkos::deep_copy(h, d_gbxs);
  for (size_t ii = 0; ii < dev.ngbxs; ++ii) {
    State& s = h(ii).state;
    s.press = a.press[ii];
    s.temp = a.temp[ii];
    s.qvap = a.qvap[ii];
    s.qcond = a.qcond[ii];
    s.wvel = {a.wvel_lo[ii], a.wvel_hi[ii]};
    s.uvel = {a.uvel_lo[ii], a.uvel_hi[ii]};
    s.vvel = {a.vvel_lo[ii], a.vvel_hi[ii]};
  }
  Kokkos::deep_copy(d_gbxs, h);
}

/* CLEO's superdroplets (AoS, Superdrop of superdrop.hpp:36-356) <-> the context's SoA */
struct SoA {
  std::vector<uint32_t> gbx;
  std::vector<double> c3, c1, c2, r, msol;
  std::vector<uint64_t> xi, id;
  cleo_b200_supers resize(const size_t n) {
    const size_t m = n ? n : 1;
    gbx.resize(m), c3.resize(m), c1.resize(m), c2.resize(m), r.resize(m), msol.resize(m);
    xi.resize(m), id.resize(m);
    return cleo_b200_supers{gbx.data(), c3.data(), c1.data(), c2.data(),
                            xi.data(),  r.data(),  msol.data(), id.data()};
  }
};
inline void upload_supers(Device& dev, const viewd_constsupers totsupers) {
  const auto h = Kokkos::create_mirror_view(totsupers);
  Kokkos::deep_copy(h, totsupers);
  SoA soa;
  const cleo_b200_supers a = soa.resize(dev.nsupers);
  for (size_t k = 0; k < dev.nsupers; ++k) {
    const Superdrop& d = h(k);
    a.sdgbxindex[k] = d.get_sdgbxindex();
    a.coord3[k] = d.get_coord3();
    a.coord1[k] = d.get_coord1();
    a.coord2[k] = d.get_coord2();
    a.xi[k] = d.get_xi();
    a.radius[k] = d.get_radius();
    a.msol[k] = d.get_msol();
    a.sdid[k] = d.sdId.get_value();
  }
  check(cleo_b200_upload_supers(dev.ctx, &a, dev.nsupers), "cleo_b200_upload_supers");
}
/* All superdroplets back into CLEO's view in the order SupersInDomain keeps them (in-domain ones
 * sorted by gridbox, then the rest), then CLEO's own sort and reference setting. */
inline void download_supers(Device& dev, const viewd_gbx d_gbxs, SupersInDomain& allsupers) {
  SoA soa;
  cleo_b200_supers a = soa.resize(dev.nsupers);
  size_t nd = 0, nt = 0;
  check(cleo_b200_download_supers(dev.ctx, &a, &nd, &nt), "cleo_b200_download_supers");
  const viewd_supers totsupers = allsupers.get_totsupers();
  if (nt != totsupers.extent(0)) fail(CLEO_ERR_CAPACITY, "superdroplet count");
  const auto h = Kokkos::create_mirror_view(totsupers);
  Kokkos::deep_copy(h, totsupers);
  for (size_t k = 0; k < nt; ++k) {
    /* the solute's properties are CLEO's single solute's (superdrop_attrs.hpp:61-259);
     * allow_nans: null superdroplets (xi = 0) leave the domain as CLEO's do */
    const SuperdropAttrs attrs(h(k).get_solute(), a.xi[k], a.radius[k], a.msol[k], true);
    h(k) = Superdrop(a.sdgbxindex[k], a.coord3[k], a.coord1[k], a.coord2[k], attrs,
                     Superdrop::IDType{(size_t)a.sdid[k]});
  }
  Kokkos::deep_copy(totsupers, h);
  allsupers.sort_and_set_totsupers(totsupers, d_gbxs);
  const auto domainsupers = allsupers.domain_supers_readonly();
  Kokkos::parallel_for(
      "cleo_b200_set_gridboxes_refs", Kokkos::RangePolicy<ExecSpace>(0, d_gbxs.extent(0)),
      KOKKOS_LAMBDA(const size_t ii) { d_gbxs(ii).supersingbx.set_refs(domainsupers); });
}

/* The per-gridbox content of CartesianMaps (cartesianmaps.hpp:188-266) as the C ABI's arrays:
 * bounds, neighbours and horizontal areas, read on the device the maps live on. */
struct GridArrays {
  std::vector<double> b[6], area;
  std::vector<uint32_t> nb[6];
  uint32_t ndims[3] = {1, 1, 1};
  cleo_b200_grid grid(const size_t ngbxs) {
    return cleo_b200_grid{(uint32_t)ngbxs, {ndims[0], ndims[1], ndims[2]},
                          b[0].data(), b[1].data(), b[2].data(), b[3].data(), b[4].data(),
                          b[5].data(), nb[0].data(), nb[1].data(), nb[2].data(), nb[3].data(),
                          nb[4].data(), nb[5].data(), area.data()};
  }
};
inline void grid_arrays(const CartesianMaps& maps, const size_t ngbxs, GridArrays& g) {
  const size_t n = ngbxs ? ngbxs : 1;
  Kokkos::View<double*> b("cleo_b200_bounds", 7 * n);
  Kokkos::View<unsigned int*> nb("cleo_b200_nghbrs", 6 * n);
  Kokkos::parallel_for(
      "cleo_b200_grid", Kokkos::RangePolicy<ExecSpace>(0, ngbxs), KOKKOS_LAMBDA(const size_t ii) {
        const auto i = (unsigned int)ii;
        const auto z = maps.coord3bounds(i), x = maps.coord1bounds(i), y = maps.coord2bounds(i);
        b(ii) = z.first, b(n + ii) = z.second, b(2 * n + ii) = x.first;
        b(3 * n + ii) = x.second, b(4 * n + ii) = y.first, b(5 * n + ii) = y.second;
        b(6 * n + ii) = maps.get_gbxarea(i);
        nb(ii) = maps.coord3backward(i), nb(n + ii) = maps.coord3forward(i);
        nb(2 * n + ii) = maps.coord1backward(i), nb(3 * n + ii) = maps.coord1forward(i);
        nb(4 * n + ii) = maps.coord2backward(i), nb(5 * n + ii) = maps.coord2forward(i);
      });
  const auto hb = Kokkos::create_mirror_view(b);
  const auto hn = Kokkos::create_mirror_view(nb);
  Kokkos::deep_copy(hb, b);
  Kokkos::deep_copy(hn, nb);
  for (int k = 0; k < 6; ++k) {
    g.b[k].assign(n, 0.0);
    g.nb[k].assign(n, 0u);
    for (size_t ii = 0; ii < ngbxs; ++ii) {
      g.b[k][ii] = hb(k * n + ii);
      g.nb[k][ii] = hn(k * n + ii);
    }
  }
  g.area.assign(n, 0.0);
  for (size_t ii = 0; ii < ngbxs; ++ii) g.area[ii] = hb(6 * n + ii);
  const auto nd = maps.get_global_ndims_hostcopy();
  for (int m = 0; m < 3; ++m) g.ndims[m] = (uint32_t)nd(m);
}

}  // namespace cleo_b200_adapter

/* MicrophysicalProcess (microphysicalprocess.hpp:45-52) carrying the B200 step's parameters:
 * those of Condensation (condensation.hpp:242-253) >> the collisions (CollCoal,
 * coalescence.hpp:133-160; CoalBuRe, coalbure.hpp:156-185; CollBu, breakup.hpp:97-123), and the
 * motion's. Its timestepping is the combined process's; its per-gridbox run_step is never
 * called, because SDMMethods is specialised for it below. */
struct B200Microphysics {
  cleo_b200_params params;

  KOKKOS_INLINE_FUNCTION unsigned int next_step(const unsigned int t) const {
    return Kokkos::min(cleo_b200_adapter::next_on(params.condstep, t),
                       cleo_b200_adapter::next_on(params.collstep, t));
  }
  KOKKOS_INLINE_FUNCTION bool on_step(const unsigned int t) const {
    return cleo_b200_adapter::on(params.condstep, t) || cleo_b200_adapter::on(params.collstep, t);
  }
  template <SDMMonitor SDMMo>
  KOKKOS_INLINE_FUNCTION subviewd_supers run_step(const TeamMember& team_member,
                                                  const unsigned int subt, subviewd_supers supers,
                                                  State& state, const SDMMo mo) const {
    return supers;
  }
};

/* Motion<GbxMaps> (superdrops/motion.hpp:32-39) carrying the motion interval; like
 * B200Microphysics it only satisfies the concept, the motion itself runs in the B200 step. */
template <GridboxMaps GbxMaps>
struct B200Motion {
  unsigned int interval;

  KOKKOS_INLINE_FUNCTION unsigned int next_step(const unsigned int t) const {
    return cleo_b200_adapter::next_on(interval, t);
  }
  KOKKOS_INLINE_FUNCTION bool on_step(const unsigned int t) const {
    return cleo_b200_adapter::on(interval, t);
  }
  KOKKOS_INLINE_FUNCTION void superdrop_coords(const unsigned int t, const GbxMaps& gbxmaps,
                                               const State& state, Superdrop& drop) const {}
  KOKKOS_INLINE_FUNCTION void superdrop_gbx(const unsigned int t, const GbxMaps& gbxmaps,
                                            Superdrop& drop) const {}
};

/* Factories in the place of CLEO's (Condensation(...) >> CollCoal(...) etc., CartesianMotion). */
inline B200Microphysics b200_microphysics(const cleo_b200_params& p) { return B200Microphysics{p}; }
template <GridboxMaps GbxMaps>
inline B200Motion<GbxMaps> b200_motion(const cleo_b200_params& p) {
  return B200Motion<GbxMaps>{p.motionstep};
}

template <Observer Obs>
class SDMMethods<CartesianMaps, B200Microphysics, B200Motion<CartesianMaps>,
                 CartesianTransportAcrossDomain, NullBoundaryConditions, Obs> {
 private:
  unsigned int couplstep;
  std::shared_ptr<cleo_b200_adapter::Device> dev;

  cleo_b200_adapter::Device& device() const {
    if (!dev->ctx) throw std::runtime_error("cleo_b200: prepare_to_timestep was not called");
    return *dev;
  }

 public:
  CartesianMaps gbxmaps;
  Obs obs;
  B200Microphysics microphys;

  /* the primary template's constructor (sdmmethods.hpp:244-250); movesupers carries the motion
   * interval, which must be the parameters' */
  SDMMethods(const unsigned int couplstep, const CartesianMaps gbxmaps,
             const B200Microphysics microphys,
             const MoveSupersInDomain<CartesianMaps, B200Motion<CartesianMaps>,
                                      CartesianTransportAcrossDomain, NullBoundaryConditions>
                 movesupers,
             const Obs obs)
      : couplstep(couplstep),
        dev(std::make_shared<cleo_b200_adapter::Device>()),
        gbxmaps(gbxmaps),
        obs(obs),
        microphys(microphys) {
    if (movesupers.next_step(0) != cleo_b200_adapter::next_on(microphys.params.motionstep, 0))
      throw std::invalid_argument("cleo_b200: the motion interval differs from the parameters'");
  }

  KOKKOS_INLINE_FUNCTION auto get_couplstep() const { return couplstep; }

  KOKKOS_INLINE_FUNCTION unsigned int next_couplstep(const unsigned int t_mdl) const {
    return ((t_mdl / couplstep) + 1) * couplstep;  // sdmmethods.hpp:274-277
  }

  /* sdmmethods.hpp:288-292, with the device context created and filled first */
  void prepare_to_timestep(const dualview_gbx gbxs, const SupersInDomain& allsupers) const {
    using namespace cleo_b200_adapter;
    Device& d = *dev;
    const auto d_gbxs = gbxs.view_device();
    d.ngbxs = d_gbxs.extent(0);
    d.nsupers = allsupers.get_totsupers_readonly().extent(0);
    if (!d.ctx) {
      GridArrays g;
      grid_arrays(gbxmaps, d.ngbxs, g);
      const cleo_b200_grid grid = g.grid(d.ngbxs);
      check(cleo_b200_create(&microphys.params, &grid, d.nsupers, &d.ctx), "cleo_b200_create");
    }
    upload_states(d, d_gbxs);
    upload_supers(d, allsupers.get_totsupers_readonly());
    obs.before_timestepping(d_gbxs, allsupers.domain_supers_readonly());
  }

  /* sdmmethods.hpp:304-309: the observers see the data run_step mirrored back */
  void at_start_step(const unsigned int t_mdl, const dualview_gbx gbxs,
                     const SupersInDomain& allsupers) const {
    obs.at_start_step(t_mdl, gbxs.view_device(), allsupers.domain_supers_readonly());
  }

  /* sdmmethods.hpp:319-332 on the GPU: every SDM step of [t_mdl, t_mdl_next) in one call */
  void run_step(const unsigned int t_mdl, const unsigned int t_mdl_next, viewd_gbx d_gbxs,
                SupersInDomain& allsupers) const {
    using namespace cleo_b200_adapter;
    Device& d = device();
    if (t_mdl % couplstep == 0) upload_states(d, d_gbxs);  // written by the coupled dynamics
    check(cleo_b200_step(d.ctx, t_mdl, t_mdl_next), "cleo_b200_step");
    cleo_b200_error e{};
    const int code = cleo_b200_status(d.ctx, &e);
    if (code != CLEO_OK)
      throw std::runtime_error("cleo_b200: the SDM step failed with status " +
                               std::to_string(code) + " (gridbox " + std::to_string(e.gbxindex) +
                               ", superdroplet " + std::to_string(e.index) + ")");
    const bool observe = obs.on_step(t_mdl_next);
    if (observe || t_mdl_next % couplstep == 0) download_states(d, d_gbxs);
    if (observe) download_supers(d, d_gbxs, allsupers);
  }

  /* the context, for calls of the C ABI beyond SDMMethods' interface (budgets, monitors,
   * output, autotuning); null before prepare_to_timestep */
  cleo_b200_ctx* context() const { return dev->ctx; }
};

#endif  // CLEO_B200_SDMMETHODS_HPP_
