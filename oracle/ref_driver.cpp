// Oracle driver: runs the reference solver's own time step, unmodified and
// compiled in place from its sources, and dumps its state so the GPU path
// can be checked against it.  Test infrastructure only.
//
// The loop mirrors the reference main() (main.cpp:84-116 plus TimeOperation,
// main.cpp:184-223): AMR::InterfaceExchange -> Body::IBConditions_Image ->
// NS_Solver::TimeMarching -> ++ts, t += dt -> ADPRule/PerformAdaptive.  Two
// harness-only settings that the reference exposes only at compile time:
//   * stage count: NS_Solver hard-wires sub_time_step = 3 (NS_Solver.H:200);
//     the subclass below sets 3 or 4 stages and the matching coefficients
//     (NS_Solver.H:204-218) through the protected members;
//   * limiter: Slopelimiter.H:20 #defines ALimiter as VanLeer; building this
//     file with -DORACLE_MINMOD redefines it to minmod (Slopelimiter.H:84-87)
//     before NS_Solver.H's flux macros are expanded in this translation unit
//     (the only one that instantiates NS_Solver::ComputeFaceFlux).
//
// Environment: IB_STEPS (default 5), IB_STAGES (3 or 4, default 4),
// IB_DUMP=<prefix> (write <prefix>_<step>.bin for the initial state and after
// each step listed by IB_DUMP_EVERY, default every step), IB_FORCES=1 (static
// body: compute wall forces each step, Body::ComptWallForce).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "Check.H"
using namespace std;  // the reference headers assume it (min/max/abs in macros)
#include "Slopelimiter.H"
#ifdef ORACLE_MINMOD
#undef ALimiter
#define ALimiter(qr, limitvalue) minvalue(limitvalue, qr, 1.0)
#endif

#include "AMR.H"
#include "AMRSpaceTime.H"
#include "Body.H"
#include "Domain.H"
#include "Mesh.H"
#include "NS_Solver.H"
#include "Pltoutput.H"
#include "TwoLevelOp.H"

extern const double Ma;

namespace {

int env_int(const char *n, int d) {
  const char *s = std::getenv(n);
  return (s && *s) ? std::atoi(s) : d;
}

class OracleSolver : public NS_Solver {
 public:
  OracleSolver(Mesh &m, Domain &d, int nbody, int stages) : NS_Solver(m, d, nbody) {
    sub_time_step = stages;
    tp.resize(stages);
    if (stages == 4) {
      tp[0] = 0.1084; tp[1] = 0.2602; tp[2] = 0.5052; tp[3] = 1.0;
    } else {
      sub_time_step = 3;
      tp.resize(3);
      tp[0] = 0.1918; tp[1] = 0.4929; tp[2] = 1.0;
    }
  }
  int stages() const { return sub_time_step; }
  double coef(int k) const { return tp[k]; }
};

// Minimal tagged binary record writer: [u32 name_len][name][u32 kind][u64 n][payload]
// kind 0 = float64, 1 = int32.
struct Dump {
  FILE *f = nullptr;
  explicit Dump(const std::string &path) { f = std::fopen(path.c_str(), "wb"); }
  ~Dump() { if (f) std::fclose(f); }
  void head(const char *name, uint32_t kind, uint64_t n) {
    uint32_t len = (uint32_t)std::strlen(name);
    std::fwrite(&len, 4, 1, f);
    std::fwrite(name, 1, len, f);
    std::fwrite(&kind, 4, 1, f);
    std::fwrite(&n, 8, 1, f);
  }
  void f64(const char *name, const std::vector<double> &v) {
    head(name, 0, v.size());
    if (!v.empty()) std::fwrite(v.data(), 8, v.size(), f);
  }
  void i32(const char *name, const std::vector<int32_t> &v) {
    head(name, 1, v.size());
    if (!v.empty()) std::fwrite(v.data(), 4, v.size(), f);
  }
};

// Every box of the z = 0 plane of every level (normal cells and 2-D ghosts),
// keyed by (level, ix, iy) so the comparison never depends on the
// reference's internal array order.
void dump_state(const std::string &path, Mesh &mesh, OracleSolver &solver,
                const std::vector<double> &forces) {
  Dump d(path);
  std::vector<int32_t> lev, ix, iy, kind, ptype, solid, infect;
  std::vector<double> prim, signdis;
  int nlev = mesh.MyCurNum();
  for (int l = 0; l < nlev; ++l) {
    DataArray<Box> &boxes = mesh.ShowLevelBox(l);
    DataArray<FlowVariables> &data = mesh.LevelDataArray(l);
    int nreal = boxes.realsize();
    int nnorm = boxes.size();
    for (int b = 0; b < nreal; ++b) {
      Box &bx = boxes[b];
      if (bx.iz() != 0) continue;
      lev.push_back(l);
      ix.push_back(bx.ix());
      iy.push_back(bx.iy());
      // 0 = normal (leaf) cell, 1 = domain ghost, 2 = block/periodic ghost,
      // 3 = other ghost (coarse/fine interface)
      int k = 3;
      if (b < nnorm) k = 0;
      else if (bx.type == Dmghost) k = 1;
      else if (bx.type == Blockghost) k = 2;
      kind.push_back(k);
      ptype.push_back((int)bx.ptype);
      solid.push_back(bx.solid ? 1 : 0);
      int inf = -1;
      if (l == nlev - 1 && mesh.Infectboxnum() > b) inf = mesh.BoxInfectIndex(b);
      infect.push_back(inf);
      signdis.push_back(bx.pair.signdis);
      FlowVariables &fv = data[b];
      prim.push_back(fv.roe);
      prim.push_back(fv.u);
      prim.push_back(fv.v);
      prim.push_back(fv.w);
      prim.push_back(fv.p);
      prim.push_back(fv.T);
      prim.push_back(fv.e);
    }
  }
  std::vector<double> scal = {t, dt, CFL_dt, (double)ts, gama, Rg, Cv, Cp, Ma, Re, Pr, qk,
                              S_over_T_ref, CFL, (double)solver.stages()};
  for (int k = 0; k < solver.stages(); ++k) scal.push_back(solver.coef(k));
  d.f64("scalars", scal);
  std::vector<double> dhv;
  for (int l = 0; l < nlev; ++l) {
    dhv.push_back(dh[l][0]);
    dhv.push_back(dh[l][1]);
    dhv.push_back(dh[l][2]);
  }
  d.f64("dh", dhv);
  std::vector<int32_t> sched;
  for (int l = 0; l < nlev; ++l) {
    sched.push_back(marching_step[l]);
    sched.push_back(average_step[l]);
    sched.push_back(prolongation_step[l]);
    sched.push_back(marching_left_step[l]);
    sched.push_back(average_left_step[l]);
    sched.push_back(prolongation_left_step[l]);
  }
  d.i32("schedule", sched);
  std::vector<int32_t> dom = {highpt.xy[0], highpt.xy[1], periodic[0] ? 1 : 0, periodic[1] ? 1 : 0,
                              (int32_t)Body::Bodynum(), nlev};
  d.i32("domain", dom);
  std::vector<double> initv = {initvar.roe, initvar.u, initvar.v, initvar.w,
                               initvar.p,   initvar.T, initvar.e};
  d.f64("initvar", initv);
  d.i32("level", lev);
  d.i32("ix", ix);
  d.i32("iy", iy);
  d.i32("kind", kind);
  d.i32("ptype", ptype);
  d.i32("solid", solid);
  d.i32("infect", infect);
  d.f64("signdis", signdis);
  d.f64("prim", prim);
  d.f64("forces", forces);
}

}  // namespace

int main(int argc, char **argv) {
  MPI_Init(&argc, &argv);
  MPI_CreateNode();
  InitSpaceParams();
  Domain p_domain(lowpt, highpt, periodic);
  Mesh mesh(p_domain, max_mesh_level);
  std::vector<Body> sphere;
  std::vector<Body> localbody;
  Body::SetBodyParams(sphere, mesh, localbody);
  AMR amr(mesh);
  Pltoutput pltfile(mesh);
  pltfile.Design_User_File();
  amr.SetupNewAMR(sphere);
  Body::ImmerseWallBoundary(mesh, sphere);

  const int stages = env_int("IB_STAGES", 4);
  OracleSolver flowsolver(mesh, p_domain, (int)sphere.size(), stages);
  amr.AllocateDataMem();
  if (env_int("IB_USER_INIT", 1)) flowsolver.InitFlow_User();
  else flowsolver.InitFlow();

  const int nsteps = env_int("IB_STEPS", 5);
  const int timed_from = env_int("IB_TIMED_FROM", 0);  // steps before this are warm-up
  const int every = env_int("IB_DUMP_EVERY", 1);
  const bool forces_on = env_int("IB_FORCES", 0) != 0;
  const char *prefix = std::getenv("IB_DUMP");
  std::vector<double> forces;
  auto do_dump = [&](int step) {
    if (!prefix) return;
    char buf[64];
    std::snprintf(buf, sizeof buf, "_%06d.bin", step);
    dump_state(std::string(prefix) + buf, mesh, flowsolver, forces);
  };
  do_dump(0);

  double loop_time = 0.0;
  long long cell_updates = 0;
  for (int s = 0; s < nsteps; ++s) {
    // leaf cells of the levels that march this step (subcycling schedule)
    long long marching_cells = 0;
    for (int l = 0; l < mesh.MyCurNum(); ++l)
      if (ts % marching_step[l] == marching_left_step[l]) marching_cells += mesh.ShowLevelBox(l).size();
    double t0 = MPI_Wtime();
    amr.InterfaceExchange();
    Body::IBConditions_Image(mesh, sphere);
    flowsolver.TimeMarching(amr);
    ++ts;
    t += dt;
    double t1 = MPI_Wtime();
    if (s >= timed_from) {
      loop_time += t1 - t0;
      cell_updates += marching_cells;
    }
    forces.clear();
    if (forces_on) {
      for (size_t b = 0; b < sphere.size(); ++b) {
        sphere[b].ComptWallForce(mesh);
        for (int k = 0; k < 3; ++k) forces.push_back(sphere[b].draglift(k));
        for (int k = 0; k < 3; ++k) forces.push_back(sphere[b].bodymoment(k));
      }
    }
    amr.ADPRule(sphere);
    if (adpflag) amr.PerformAdaptive(sphere);
    adpflag = false;
    if (prefix && (ts % every == 0 || s == nsteps - 1)) do_dump(ts);
  }
  std::printf("ORACLE_RESULT {\"steps\": %d, \"loop_seconds\": %.9f, \"cell_updates\": %lld, "
              "\"cell_updates_per_s\": %.6e, \"t\": %.17g, \"dt\": %.17g}\n",
              nsteps - timed_from, loop_time, cell_updates,
              loop_time > 0 ? (double)cell_updates / loop_time : 0.0, t, dt);
  MPI_Finalize();
  return 0;
}
