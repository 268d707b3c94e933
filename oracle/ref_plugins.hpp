/*
 * ref_plugins.hpp — CLEO's own plug-ins selected at run time (TEST INFRASTRUCTURE ONLY).
 *
 * Shared by the harnesses that build CLEO's objects from its unmodified sources against the
 * Kokkos-API shim (ref_harness.cpp, adapter_harness.cpp). The only project code here is dispatch:
 * small structs that satisfy the reference's VelocityFormula / PairProbability / PairEnactX /
 * NFragments / CoalBuReFlag concepts by forwarding to the reference's own implementations, so
 * that one instantiation of SDMMethods serves every plug-in combination a cleo_b200_params
 * selects; the microphysics is built the way CollCoal/CollBu/CoalBuRe build it
 * (coalescence.hpp:149-160, breakup.hpp:111-123, coalbure.hpp:173-185) and Condensation through
 * its own factory (condensation.hpp:242-253); the CartesianMaps are filled like
 * set_cartesian_maps (createcartesianmaps.cpp:143-252).
 */
#ifndef CLEO_B200_ORACLE_REF_PLUGINS_HPP_
#define CLEO_B200_ORACLE_REF_PLUGINS_HPP_

#include <functional>

#include "../include/cleo_b200.h"
#include "cartesiandomain/cartesianmaps.hpp"
#include "cartesiandomain/movement/cartesian_motion.hpp"
#include "cartesiandomain/movement/cartesian_movement.hpp"
#include "gridboxes/boundary_conditions.hpp"
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
#include "superdrops/microphysicalprocess.hpp"
#include "superdrops/terminalvelocity.hpp"

/* ---- run-time selection of the reference's plug-ins ---- */
struct AnyTV {
  int kind = CLEO_TV_NULL;
  KOKKOS_FUNCTION double operator()(const Superdrop& d) const {
    switch (kind) {
      case CLEO_TV_SIMMEL: return SimmelTerminalVelocity{}(d);
      case CLEO_TV_ROGERSYAU: return RogersYauTerminalVelocity{}(d);
      case CLEO_TV_ROGERSGK: return RogersGKTerminalVelocity{}(d);
      default: return NullTerminalVelocity{}(d);
    }
  }
};

struct AnyProb {
  int kind;
  GolovinProb golovin;
  LongHydroProb longhydro;
  ConstProb constprob;
  AnyProb(int k, double coaleff, double kernel)
      : kind(k), golovin(), longhydro(coaleff), constprob(kernel) {}
  KOKKOS_FUNCTION double operator()(const Superdrop& a, const Superdrop& b, const double DELT,
                                    const double VOLUME) const {
    switch (kind) {
      case CLEO_PROB_GOLOVIN: return golovin(a, b, DELT, VOLUME);
      case CLEO_PROB_LONG: return longhydro(a, b, DELT, VOLUME);
      default: return constprob(a, b, DELT, VOLUME);
    }
  }
};

struct AnyNFrags {
  int kind;
  ConstNFrags cnf;
  CollisionKineticEnergyNFrags<AnyTV> cke;
  AnyNFrags(int k, double nfrags, int tv) : kind(k), cnf(nfrags), cke(AnyTV{tv}) {}
  KOKKOS_FUNCTION double operator()(const Superdrop& a, const Superdrop& b) const {
    return kind == CLEO_NFRAGS_CONST ? cnf(a, b) : cke(a, b);
  }
};

struct AnyFlag {
  int kind;
  StraubCoalBuReFlag<AnyTV> straub;
  TSCoalBuReFlag<AnyTV> ts;
  SUCoalBuReFlag<AnyTV> su;
  ConstCoalBuReFlag cst;
  AnyFlag(int k, int tv, double coaleff)
      : kind(k), straub(AnyTV{tv}), ts(AnyTV{tv}), su(AnyTV{tv}), cst(coaleff) {}
  KOKKOS_FUNCTION unsigned int operator()(const double phi, const Superdrop& a,
                                          const Superdrop& b) const {
    switch (kind) {
      case CLEO_FLAG_STRAUB: return straub(phi, a, b);
      case CLEO_FLAG_TESTIKSTRAUB: return ts(phi, a, b);
      case CLEO_FLAG_SZAKALLURBICH: return su(phi, a, b);
      default: return cst(phi, a, b);
    }
  }
};

struct AnyEnact {
  int kind;
  DoCoalescence coal;
  DoBreakup<AnyNFrags> bu;
  DoCoalBuRe<AnyNFrags, AnyFlag> coalbure;
  AnyEnact(int k, AnyNFrags nf, AnyFlag fl) : kind(k), coal(), bu(nf), coalbure(nf, fl) {}
  KOKKOS_FUNCTION size_t operator()(Superdrop& d1, Superdrop& d2, const double prob,
                                    const double phi_coll, const double phi_out) const {
    switch (kind) {
      case CLEO_ENACT_COALESCENCE: return coal(d1, d2, prob, phi_coll, phi_out);
      case CLEO_ENACT_BREAKUP: return bu(d1, d2, prob, phi_coll, phi_out);
      default: return coalbure(d1, d2, prob, phi_coll, phi_out);
    }
  }
};

using Colls = ConstTstepMicrophysics<DoCollisions<AnyProb, AnyEnact>>;
using Cond = decltype(Condensation(1u, std::function<double(unsigned int)>{}, false, 1, 0.0, 0.0,
                                   0.0, std::function<double(double)>{}));
using Microphys = CombinedMicrophysicalProcess<Cond, Colls>;
using MotionT = PredCorrMotion<CartesianMaps, AnyTV, CartesianCheckBounds>;

/* Condensation >> collisions of the given parameters */
inline Microphys ref_microphysics(const cleo_b200_params& P) {
  const Cond cond = Condensation(
      P.condstep, [P](unsigned int) { return P.cond_delt; }, P.do_alter_thermo != 0,
      P.maxniters, P.rtol, P.atol, 0.0, [P](double) { return P.cond_minsubdelt; });
  const AnyNFrags nf(P.nfrags_kind, P.nfrags, P.nfrags_tv);
  const AnyFlag fl(P.flag_kind, P.flag_tv, P.flag_coaleff);
  const AnyEnact enact(P.coll_enact, nf, fl);
  const AnyProb prob(P.coll_prob, P.coaleff, P.const_kernel);
  const Colls colls(P.collstep, DoCollisions<AnyProb, AnyEnact>(P.coll_delt, prob, enact, P.seed));
  return cond >> colls;
}

/* CartesianMotion (cartesian_motion.hpp:60-66) of the given parameters */
inline MotionT ref_motion(const cleo_b200_params& P) {
  return CartesianMotion(P.motionstep, [P](unsigned int) { return P.motion_delt; },
                         AnyTV{P.motion_tv});
}

/* CartesianMaps for an undecomposed domain from the given bounds and neighbours (the states
 * carry the gridbox volumes: the volume map is 0, or `volumes` where it is given) */
inline CartesianMaps ref_cartesian_maps(const cleo_b200_grid* g, const double* volumes) {
  CartesianMaps maps;
  const size_t sz = (size_t)g->ngbxs + 1;
  const auto h3 = kokkos_pairmap::HostMirror(sz), h1 = kokkos_pairmap::HostMirror(sz),
             h2 = kokkos_pairmap::HostMirror(sz);
  const auto b3 = kokkos_uintmap::HostMirror(sz), f3 = kokkos_uintmap::HostMirror(sz),
             b1 = kokkos_uintmap::HostMirror(sz), f1 = kokkos_uintmap::HostMirror(sz),
             b2 = kokkos_uintmap::HostMirror(sz), f2 = kokkos_uintmap::HostMirror(sz);
  const auto areas = kokkos_dblmaph(sz), vols = kokkos_dblmaph(sz);
  const auto oob = LIMITVALUES::oob_gbxindex;
  const Kokkos::pair<double, double> nullb{LIMITVALUES::llim, LIMITVALUES::ulim};
  h3.insert(oob, nullb); h1.insert(oob, nullb); h2.insert(oob, nullb);
  b3.insert(oob, oob); f3.insert(oob, oob); b1.insert(oob, oob);
  f1.insert(oob, oob); b2.insert(oob, oob); f2.insert(oob, oob);
  areas.insert(oob, 0.0); vols.insert(oob, 0.0);
  for (unsigned int i = 0; i < g->ngbxs; ++i) {
    h3.insert(i, {g->coord3lo[i], g->coord3hi[i]});
    h1.insert(i, {g->coord1lo[i], g->coord1hi[i]});
    h2.insert(i, {g->coord2lo[i], g->coord2hi[i]});
    b3.insert(i, g->back3[i]); f3.insert(i, g->fwd3[i]);
    b1.insert(i, g->back1[i]); f1.insert(i, g->fwd1[i]);
    b2.insert(i, g->back2[i]); f2.insert(i, g->fwd2[i]);
    const double area = g->gbxarea ? g->gbxarea[i]
                                   : (g->coord1hi[i] - g->coord1lo[i]) *
                                         (g->coord2hi[i] - g->coord2lo[i]);
    areas.insert(i, area);
    vols.insert(i, volumes ? volumes[i] : 0.0);
  }
  maps.set_coord3bounds_via_copy(h3);
  maps.set_coord1bounds_via_copy(h1);
  maps.set_coord2bounds_via_copy(h2);
  maps.set_back_coord3nghbr_via_copy(b3);
  maps.set_forward_coord3nghbr_via_copy(f3);
  maps.set_back_coord1nghbr_via_copy(b1);
  maps.set_forward_coord1nghbr_via_copy(f1);
  maps.set_back_coord2nghbr_via_copy(b2);
  maps.set_forward_coord2nghbr_via_copy(f2);
  maps.set_gbxareas_map(areas);
  maps.set_gbxvolumes_map(vols);
  auto hnd = Kokkos::create_mirror_view(maps.get_global_ndims());
  for (int m = 0; m < 3; ++m) hnd(m) = g->ndims[m];
  maps.set_global_ndims_via_copy(hnd);
  return maps;
}

#endif  // CLEO_B200_ORACLE_REF_PLUGINS_HPP_
