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
// IB_TAG_SERVER=<dir> (runtime regrids of the case file: write the state the
// tag server decides from to <dir>/state_<ts>.bin before each regrid),
// IB_DUMP=<prefix> (write <prefix>_<step>.bin for the initial state and after
// each step listed by IB_DUMP_EVERY, default every step, or only after the
// step counts IB_DUMP_AT lists), IB_FORCES=1 (static
// body: compute wall forces each step, Body::ComptWallForce), IB_FORCE_LOG=<file>
// (the per-step force history), IB_RANKS=N (the reference's shared-memory
// mode with N ranks on one node; the shim in mpi_shim/ forks them),
// IB_PLT=<prefix> (the reference's Tecplot solution file of the final state).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <fstream>
#include <iostream>
#include <sstream>
#include <unistd.h>

// Test-infrastructure access: the dump below reads the reference's private
// AMR pair lists, boundary values and immersed-boundary records.  Standard
// headers are included above so only the reference's own classes see this.
#define private public
#define protected public

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
#ifdef ORACLE_BINDING
#include "ibgpu_ns_solver.H"
#endif

extern const double Ma;
extern double p_ref, area_ref, shear_ref;
extern double dt00;  // time since the bodies last moved (Body.cpp)
extern FILE *g_oracle_tag_dump;  // defined by the case file (tag dump hook)
extern int g_oracle_tag_pass;

namespace {

int env_int(const char *n, int d) {
  const char *s = std::getenv(n);
  return (s && *s) ? std::atoi(s) : d;
}

#ifdef ORACLE_BINDING
// the binding build: the same solver with the reference-side GPU binding
// underneath, stepping on the GPU once on_gpu is set (IB_BINDING_STEP)
typedef GpuNS_Solver SolverBase;
#ifdef ORACLE_MINMOD
const int kLimiter = IBGPU_LIM_MINMOD;
#else
const int kLimiter = IBGPU_LIM_VANLEER;
#endif
#else
typedef NS_Solver SolverBase;
#endif

class OracleSolver : public SolverBase {
 public:
  OracleSolver(Mesh &m, Domain &d, int nbody, int stages) : SolverBase(m, d, nbody) {
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
#ifdef ORACLE_BINDING
  bool on_gpu = false;
  void TimeMarching(AMR &amr) {
    if (on_gpu) GpuNS_Solver::TimeMarching(amr);
    else NS_Solver::TimeMarching(amr);
  }
#endif
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

AMR *g_amr = nullptr;
std::vector<Body> *g_bodies = nullptr;

inline void put_pos(std::vector<int32_t> &v, Mesh &mesh, int l, int b) {
  if (b < 0) {
    v.push_back(INT32_MIN);
    v.push_back(INT32_MIN);
    return;
  }
  Box &bx = mesh.ShowLevelBox(l)[b];
  v.push_back(bx.ix());
  v.push_back(bx.iy());
}

// Coarse/fine pairs (AMRLevel::f_res_ghost, f_pro_ghost, g_pro), positions
// of the coarse box and its four z = 0 sons in Point_iterator_2d order.
void dump_interfaces(Dump &d, Mesh &mesh, AMR &amr) {
  std::vector<int32_t> res, pro;
  int nlev = mesh.MyCurNum();
  for (int l = 0; l + 1 < nlev; ++l) {
    AMRLevel &al = amr.m_level[l];
    for (int ig = 0; ig < ighost; ++ig) {
      DataArray<CtoFPair> &lst = al.f_res_ghost[ig];
      for (int i = 0; i < lst.size(); ++i) {
        res.push_back(l);
        res.push_back(ig);
        put_pos(res, mesh, l, lst[i].ci);
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) put_pos(res, mesh, l + 1, lst[i].fi.son[a][b][0]);
      }
    }
    for (int i = 0; i < al.f_pro_ghost.size(); ++i) {
      pro.push_back(l);
      pro.push_back(0);
      put_pos(pro, mesh, l, al.f_pro_ghost[i].ci);
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) put_pos(pro, mesh, l + 1, al.f_pro_ghost[i].fi.son[a][b][0]);
    }
    for (int i = 0; i < al.g_pro.size(); ++i) {
      CtoFPair &cfp = al.level_pro_ghost[al.g_pro[i]];
      pro.push_back(l);
      pro.push_back(1);
      put_pos(pro, mesh, l, cfp.ci);
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) put_pos(pro, mesh, l + 1, cfp.fi.son[a][b][0]);
    }
  }
  d.i32("cf_res", res);
  d.i32("cf_pro", pro);
}

// Domain ghosts in BCBoxTreat order (BCValues.H:51-188) and the face values.
void dump_boundaries(Dump &d, Mesh &mesh, OracleSolver &solver) {
  std::vector<int32_t> bc;
  std::vector<double> nmv;
  int nlev = mesh.MyCurNum();
  for (int l = 0; l < nlev; ++l) {
    DataArray<Domainghost> &dmg = mesh.MeshGhostArray(l);
    for (int i = 0; i < dmg.size(); ++i) {
      int f0 = dmg[i].nbface;
      bc.push_back(l);
      put_pos(bc, mesh, l, dmg[i].cell);
      put_pos(bc, mesh, l, dmg[i].refcell);
      bc.push_back(f0);
      bc.push_back(mesh.m_dm.facetype[f0]);
      bc.push_back(mesh.m_dm.facedir[f0][2] != 0 ? 1 : 0);
      bc.push_back(mesh.ShowLevelBox(l)[dmg[i].cell].iz());
      nmv.push_back(dmg[i].nmv[0]);
      nmv.push_back(dmg[i].nmv[1]);
      nmv.push_back(dmg[i].nmv[2]);
    }
  }
  d.i32("bc", bc);
  d.f64("bc_nmv", nmv);
  BCValues &B = solver.meshbc;
  std::vector<double> fv;
  for (size_t f = 0; f < B.facevar.size(); ++f) {
    FlowVariables &v = B.facevar[f];
    double r[7] = {v.roe, v.u, v.v, v.w, v.p, v.T, v.e};
    fv.insert(fv.end(), r, r + 7);
  }
  d.f64("facevar", fv);
  std::vector<double> bs = {B.backpressure, inlet_flow_angle};
  d.f64("bc_scalars", bs);
}

// Immersed-boundary cells processed by Body::IBConditions_Image
// (Body.cpp:1361-1496) and the surface patches of Body::ComptWallForce
// (Body.cpp:439-558).
void dump_body(Dump &d, Mesh &mesh, std::vector<Body> &bodies) {
  std::vector<int32_t> ib, pat;
  std::vector<double> ibf, patf, bodyf;
  int last = mesh.MyCurNum() - 1;
  DataArray<IBCell> &mdis = mesh.ibarray();
  for (int i = 0; i < mdis.size(); ++i) {
    IBCell &c = mdis[i];
    if (!(mesh.m_level[last].m_box.isnormal(c.ci) && c.mynode == node)) continue;
    BoxtoWall &w = mesh.m_level[last].m_box[c.ci].pair;
    put_pos(ib, mesh, last, c.ci);
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int k = 0; k < 2; ++k) put_pos(ib, mesh, last, c.hgc.intpcell[a][b][k]);
    ib.push_back(w.body);
    ib.push_back(w.patch);
    Pointxyz patv;
    bodies[w.body].Surface_Point_Velocity(c.hgc.attach_pt, patv);
    Pointxyz &nv = bodies[w.body].patch[w.patch].nv;
    ibf.push_back(w.signdis);
    ibf.push_back(c.hgc.hgdis);
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int k = 0; k < 2; ++k) ibf.push_back(c.hgc.intpcoef[a][b][k]);
    for (int k = 0; k < 3; ++k) ibf.push_back(nv[k]);
    for (int k = 0; k < 3; ++k) ibf.push_back(patv[k]);
  }
  for (size_t bi = 0; bi < bodies.size(); ++bi) {
    Body &B = bodies[bi];
    for (int k = 0; k < 3; ++k) bodyf.push_back(B.bodycenter[k]);
    for (int i = 0; i < B.patch.size(); ++i) {
      Surfpatch &P = B.patch[i];
      if (P.node != node) continue;
      pat.push_back((int32_t)bi);
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          for (int k = 0; k < 2; ++k) put_pos(pat, mesh, last, P.hgc.intpcell[a][b][k]);
      for (int k = 0; k < 3; ++k) patf.push_back(P.pc[k]);
      for (int k = 0; k < 3; ++k) patf.push_back(P.nv[k]);
      patf.push_back(P.area);
      patf.push_back(P.hgc.hgdis);
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          for (int k = 0; k < 2; ++k) patf.push_back(P.hgc.intpcoef[a][b][k]);
      Pointxyz patv;
      B.Surface_Point_Velocity(P.pc, patv);
      for (int k = 0; k < 3; ++k) patf.push_back(patv[k]);
    }
  }
  d.i32("ib", ib);
  d.f64("ib_f", ibf);
  d.i32("patch", pat);
  d.f64("patch_f", patf);
  bodyf.push_back(p_ref);
  bodyf.push_back(area_ref);
  bodyf.push_back(shear_ref);
  bodyf.push_back(L_ref);
  bodyf.push_back(mu);
  d.f64("body_f", bodyf);
}

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
  scal.push_back((double)dt_var_step);
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
  dump_interfaces(d, mesh, *g_amr);
  dump_boundaries(d, mesh, solver);
  dump_body(d, mesh, *g_bodies);
}

}  // namespace

int main(int argc, char **argv) {
  MPI_Init(&argc, &argv);
  MPI_CreateNode();
  // IB_RANKS=N runs the reference's own shared-memory mode with N ranks: the
  // step (the reference's, or the binding's with rank 0 driving the GPU),
  // dumps (written by rank 0) and force logs; the harness hooks that write
  // from inside the case file or dump the binding's lists need one rank
  if (nprocs > 1 && (std::getenv("IB_TAG_DUMP") || std::getenv("IB_TAG_SERVER") ||
                     std::getenv("IB_BINDING_LISTS") || std::getenv("IB_BINDING_TAGCHECK"))) {
    if (nrank == 0) std::fprintf(stderr, "tag dumps, tag server and binding lists need one rank\n");
    MPI_Abort(MPI_COMM_WORLD, 5);
  }
  InitSpaceParams();
  Domain p_domain(lowpt, highpt, periodic);
  Mesh mesh(p_domain, max_mesh_level);
  std::vector<Body> sphere;
  std::vector<Body> localbody;
  Body::SetBodyParams(sphere, mesh, localbody);
  AMR amr(mesh);
  Pltoutput pltfile(mesh);
  pltfile.Design_User_File();
  // IB_TAG_DUMP=<file>: record the case's TagtheBox decisions, 9 doubles per
  // normal box (level, ix, iy, centre x, centre y, signdis, tag, detag,
  // pass): pass 0 while the initial mesh is built (refinement requested
  // level by level, every box of the level being judged is a leaf), pass 1
  // re-judging the finished mesh with refinement and coarsening requested
  const char *tagpath = std::getenv("IB_TAG_DUMP");
  if (tagpath) {
    g_oracle_tag_dump = std::fopen(tagpath, "wb");
    g_oracle_tag_pass = 0;
  }
  amr.SetupNewAMR(sphere);
  Body::ImmerseWallBoundary(mesh, sphere);
  g_amr = &amr;
  g_bodies = &sphere;

  const int stages = env_int("IB_STAGES", 4);
  OracleSolver flowsolver(mesh, p_domain, (int)sphere.size(), stages);
  amr.AllocateDataMem();
  if (env_int("IB_USER_INIT", 1)) flowsolver.InitFlow_User();
  else flowsolver.InitFlow();

  if (tagpath) {
    g_oracle_tag_pass = 1;
    for (int l = 0; l < mesh.MyCurNum(); ++l) {
      amr.m_level[l].torefine = true;
      amr.m_level[l].toderefine = l >= 1;
      amr.TagtheBox(l, sphere);
      amr.m_level[l].torefine = false;
      amr.m_level[l].toderefine = false;
      amr.m_level[l].Inittag();
    }
    std::fclose(g_oracle_tag_dump);
    g_oracle_tag_dump = nullptr;
  }

#ifdef ORACLE_BINDING
  // IB_BINDING_LISTS=<file>: the lists and case constants the reference-side
  // binding (ibgpu_ns_solver.H) hands to the C ABI for this mesh and state,
  // and the status of ibgpu_create with them
  if (const char *bl = std::getenv("IB_BINDING_LISTS")) {
    IbgpuLists L;
    IbgpuAdapter::Flatten(mesh, amr, sphere, flowsolver, L);
    const ibgpu_case c = IbgpuAdapter::MakeCase(flowsolver, kLimiter, IBGPU_FP64);
    std::vector<int32_t> cw(sizeof c / 4);
    std::memcpy(cw.data(), &c, sizeof c);
    ibgpu_ctx *ctx = nullptr;
    const int rc = ibgpu_create(&c, &ctx);
    if (ctx) ibgpu_destroy(ctx);
    Dump d(bl);
    d.i32("level", L.level);
    d.i32("ix", L.ix);
    d.i32("iy", L.iy);
    d.i32("flags", std::vector<int32_t>(L.flags.begin(), L.flags.end()));
    d.f64("prim", L.prim);
    d.i32("res", L.res);
    d.i32("pro", L.pro);
    d.i32("bc", L.bc);
    d.f64("bc_nmv", L.bc_nmv);
    d.f64("facevar", L.facevar);
    d.f64("bc_scalars", std::vector<double>{L.backpressure, L.inlet_flow_angle});
    d.i32("ib", L.ib_cell);
    d.f64("ib_f", L.ib_cellf);
    d.i32("patch", L.patch);
    d.f64("patch_f", L.patchf);
    d.f64("body_center", L.body_center);
    d.i32("case", cw);
    d.i32("create_rc", std::vector<int32_t>{rc});
    // the boxes the binding's TagLevel judges, per level
    std::vector<int32_t> tl, tx, ty, tb;
    std::vector<double> txc, tyc, tsd;
    for (int l = 0; l < mesh.MyCurNum(); ++l) {
      IbgpuAdapter::TagBoxes T;
      IbgpuAdapter::GatherTagBoxes(mesh, amr, l, T);
      tl.insert(tl.end(), T.level.begin(), T.level.end());
      tx.insert(tx.end(), T.ix.begin(), T.ix.end());
      ty.insert(ty.end(), T.iy.begin(), T.iy.end());
      tb.insert(tb.end(), T.box.begin(), T.box.end());
      txc.insert(txc.end(), T.xc.begin(), T.xc.end());
      tyc.insert(tyc.end(), T.yc.begin(), T.yc.end());
      tsd.insert(tsd.end(), T.signdis.begin(), T.signdis.end());
    }
    d.i32("tag_level", tl);
    d.i32("tag_ix", tx);
    d.i32("tag_iy", ty);
    d.i32("tag_box", tb);
    d.f64("tag_xc", txc);
    d.f64("tag_yc", tyc);
    d.f64("tag_signdis", tsd);
  }
  // IB_BINDING_TAGCHECK=<dir>: for every level and every request the regrid
  // can make of it (refine only, coarsen only, both), the case's TagtheBox
  // decisions (tag dump rows, pass 2 + 3 * level + request) and the
  // refine / coarsen flags of the rule the binding's TagLevel hands the GPU
  // for that level (IbgpuAdapter::LevelRule of the case rule in
  // <dir>/rule.bin), one row (pass, level, torefine, toderefine) per request
  const char *tc = std::getenv("IB_BINDING_TAGCHECK");
  if (tc && *tc) {
    const std::string dir(tc);
    ibgpu_tag_rule base;
    FILE *rf = std::fopen((dir + "/rule.bin").c_str(), "rb");
    if (!rf || std::fread(&base, sizeof base, 1, rf) != 1) {
      std::fprintf(stderr, "IB_BINDING_TAGCHECK: cannot read rule.bin\n");
      return 4;
    }
    std::fclose(rf);
    g_oracle_tag_dump = std::fopen((dir + "/tags.bin").c_str(), "wb");
    std::vector<int32_t> flags;
    const int req[3][2] = {{1, 0}, {0, 1}, {1, 1}};
    for (int l = 0; l < mesh.MyCurNum(); ++l)
      for (int c = 0; c < 3; ++c) {
        for (int k = 0; k < mesh.MyCurNum(); ++k) {
          amr.m_level[k].torefine = false;
          amr.m_level[k].toderefine = false;
        }
        amr.m_level[l].torefine = req[c][0] != 0;
        amr.m_level[l].toderefine = req[c][1] != 0;
        g_oracle_tag_pass = 2 + 3 * l + c;
        amr.TagtheBox(l, sphere);
        const ibgpu_tag_rule lr = IbgpuAdapter::LevelRule(base, amr, l);
        flags.insert(flags.end(), {g_oracle_tag_pass, l, lr.torefine[l], lr.toderefine[l]});
        amr.m_level[l].torefine = false;
        amr.m_level[l].toderefine = false;
        amr.m_level[l].Inittag();
        amr.m_level[l].taggedbox.clear();
      }
    std::fclose(g_oracle_tag_dump);
    g_oracle_tag_dump = nullptr;
    Dump d(dir + "/levelrule.bin");
    d.i32("levelrule", flags);
  }
#endif

  // IB_BINDING_STEP=1: the loop steps through the binding on the GPU (FP64
  // build) instead of the reference's own step; state read back for dumps
  // and regrids, forces from the device
#ifdef ORACLE_BINDING
  const bool gpu_step = env_int("IB_BINDING_STEP", 0) != 0;
  auto gpu_check = [](int rc, const char *what) {
    if (rc == IBGPU_OK) return;
    std::fprintf(stderr, "%s: %s (%s)\n", what, ibgpu_errstr(rc), ibgpu_last_error());
    std::exit(3);
  };
  if (gpu_step) {
    // IB_BINDING_PRECISION: IBGPU_FP64 (default), IBGPU_FP64_EXACT or IBGPU_MIXED;
    // IB_BINDING_DEVICE_DISTANCE=0: the reference's own wall-distance passes
    // for moving bodies (default: the device's); IB_BINDING_DISTCHECK=1: both,
    // the boxes that differ counted
    flowsolver.SetDeviceWallDistances(env_int("IB_BINDING_DEVICE_DISTANCE", 1) != 0,
                                      env_int("IB_BINDING_DISTCHECK", 0) != 0);
    gpu_check(flowsolver.Create(kLimiter, env_int("IB_BINDING_PRECISION", IBGPU_FP64)),
              "ibgpu_create");
    gpu_check(flowsolver.Upload(amr, sphere), "upload");
    flowsolver.on_gpu = true;
  }
#else
  const bool gpu_step = false;
#endif

  const int nsteps = env_int("IB_STEPS", 5);
  const int timed_from = env_int("IB_TIMED_FROM", 0);  // steps before this are warm-up
  const int every = env_int("IB_DUMP_EVERY", 1);
  // IB_DUMP_AT=<a,b,...>: dump only after these step counts (0 = the initial
  // state) instead of every IB_DUMP_EVERY steps
  std::vector<int> dump_at;
  if (const char *at = std::getenv("IB_DUMP_AT")) {
    std::stringstream ss(at);
    std::string item;
    while (std::getline(ss, item, ',')) if (!item.empty()) dump_at.push_back(std::atoi(item.c_str()));
  }
  auto dump_now = [&](int step, bool last) {
    if (!dump_at.empty()) return std::find(dump_at.begin(), dump_at.end(), step) != dump_at.end();
    return step == 0 || step % every == 0 || last;
  };
  const bool forces_on = env_int("IB_FORCES", 0) != 0;
  const char *prefix = std::getenv("IB_DUMP");
  // IB_FORCE_LOG=<file>: per step ts, t, dt and the forces/moments of every
  // body (6 doubles each) as raw doubles, the Cl/Cd history of a run
  const char *force_log = std::getenv("IB_FORCE_LOG");
  FILE *flog = (force_log && nrank == 0) ? std::fopen(force_log, "wb") : nullptr;
  std::vector<double> forces;
  auto do_dump = [&](int step) {
    if (!prefix) return;
#ifdef ORACLE_BINDING
    if (gpu_step) gpu_check(flowsolver.Download(), "download");
#endif
    char buf[64];
    std::snprintf(buf, sizeof buf, "_%06d.bin", step);
    MPI_Barrier(MPI_COMM_WORLD);  // every rank's share of the arrays written
    if (nrank == 0) dump_state(std::string(prefix) + buf, mesh, flowsolver, forces);
    MPI_Barrier(MPI_COMM_WORLD);
  };
  if (dump_now(0, false)) do_dump(0);

  // loop_time: the timed steps (motion and re-immersion, the step); the
  // regrids between them (tagging, mesh adaptation and, through the binding,
  // the download before and the upload after) in regrid_time
  double loop_time = 0.0, move_time = 0.0, regrid_time = 0.0;
  double rg_tag = 0.0, rg_download = 0.0, rg_adapt = 0.0, rg_upload = 0.0;  // regrid parts
#ifdef ORACLE_BINDING
  IbgpuUploadTimes rg_up;  // the upload's parts over the timed regrids
#endif
  long long cell_updates = 0;
  for (int s = 0; s < nsteps; ++s) {
    // leaf cells of the levels that march this step (subcycling schedule)
    long long marching_cells = 0;
    for (int l = 0; l < mesh.MyCurNum(); ++l)
      if (ts % marching_step[l] == marching_left_step[l]) marching_cells += mesh.ShowLevelBox(l).size();
    MPI_Barrier(MPI_COMM_WORLD);  // the timed step spans every rank's share
    double t0 = MPI_Wtime();
    if (!gpu_step) {  // the GPU step runs both ghost fills itself
      amr.InterfaceExchange();
      Body::IBConditions_Image(mesh, sphere);
    }
#ifdef ORACLE_BINDING
    else if (moveflag) {
      // the moving-body part of IBConditions_Image through the binding
      const double tm0 = MPI_Wtime();
      gpu_check(flowsolver.MoveBodies(sphere, dt00), "move bodies");
      if (s >= timed_from) move_time += MPI_Wtime() - tm0;
    }
#endif
    flowsolver.TimeMarching(amr);
    ++ts;
    t += dt;
    MPI_Barrier(MPI_COMM_WORLD);
    double t1 = MPI_Wtime();
    if (s >= timed_from) {
      loop_time += t1 - t0;
      cell_updates += marching_cells;
    }
    forces.clear();
#ifdef ORACLE_BINDING
    if (forces_on && gpu_step) gpu_check(flowsolver.WallForces(forces), "ibgpu_wall_forces");
#endif
    if (forces_on && !gpu_step) {
      for (size_t b = 0; b < sphere.size(); ++b) {
        sphere[b].ComptWallForce(mesh);
        for (int k = 0; k < 3; ++k) forces.push_back(sphere[b].draglift(k));
        for (int k = 0; k < 3; ++k) forces.push_back(sphere[b].bodymoment(k));
      }
    }
    if (flog) {
      const double head[3] = {(double)ts, t, dt};
      std::fwrite(head, sizeof(double), 3, flog);
      if (!forces.empty()) std::fwrite(forces.data(), sizeof(double), forces.size(), flog);
    }
    MPI_Barrier(MPI_COMM_WORLD);
    const double tr0 = MPI_Wtime();
    const bool timed_regrid = s >= timed_from && s + 1 < nsteps;
    amr.ADPRule(sphere);
    const double tr1 = MPI_Wtime();
    double tr2 = tr1, tr3 = tr1;
#ifdef ORACLE_BINDING
    if (adpflag && gpu_step) gpu_check(flowsolver.Download(), "download");
    tr2 = tr3 = MPI_Wtime();
#endif
    if (adpflag) {
      // a tag server decides from the state it sees here (case file)
      const char *server = std::getenv("IB_TAG_SERVER");
      if (server && *server) {
        const std::string path = std::string(server) + "/state_" + std::to_string(ts) + ".bin";
        dump_state(path + ".part", mesh, flowsolver, forces);
        std::rename((path + ".part").c_str(), path.c_str());
      }
      amr.PerformAdaptive(sphere);
      tr3 = MPI_Wtime();
#ifdef ORACLE_BINDING
      const IbgpuUploadTimes u0 = ibgpu_upload_times();
      if (gpu_step) gpu_check(flowsolver.Upload(amr, sphere), "upload");
      if (timed_regrid) {
        const IbgpuUploadTimes &u1 = ibgpu_upload_times();
        rg_up.flatten += u1.flatten - u0.flatten;
        rg_up.lists += u1.lists - u0.lists;
        rg_up.wall_geometry += u1.wall_geometry - u0.wall_geometry;
        rg_up.wall_pack += u1.wall_pack - u0.wall_pack;
        rg_up.wall_device += u1.wall_device - u0.wall_device;
        rg_up.rows_map += u1.rows_map - u0.rows_map;
      }
#endif
    }
    MPI_Barrier(MPI_COMM_WORLD);
    if (timed_regrid) {
      const double tr4 = MPI_Wtime();
      regrid_time += tr4 - tr0;
      if (adpflag) {
        rg_tag += tr1 - tr0;
        rg_download += tr2 - tr1;
        rg_adapt += tr3 - tr2;
        rg_upload += tr4 - tr3;
      }
    }
    adpflag = false;
    if (prefix && dump_now(ts, s == nsteps - 1)) do_dump(ts);
  }
  if (flog) std::fclose(flog);
  // IB_PLT=<prefix>: the reference's own Tecplot solution writer
  // (Pltoutput::Output_Soln_Nobody, <prefix>-<ts>.plt) on the final state,
  // read back from the device first when the binding steps
  if (const char *plt = std::getenv("IB_PLT")) {
#ifdef ORACLE_BINDING
    if (gpu_step) gpu_check(flowsolver.Download(), "download");
#endif
    pltfile.Output_Soln_Nobody(plt);
  }
  std::string phases = "{}", rphases;
  {
    // the timed regrids' parts on rank 0: tagging (ADPRule), reading the
    // device state back, the reference's PerformAdaptive, the upload
    char buf[256];
    std::snprintf(buf, sizeof buf,
                  "{\"tag\": %.6f, \"download\": %.6f, \"adapt\": %.6f, \"upload\": %.6f",
                  rg_tag, rg_download, rg_adapt, rg_upload);
    rphases = buf;
#ifdef ORACLE_BINDING
    // the upload's parts over the timed regrids (rank 0): the cell rows and
    // lists flattened, the library's uploads, the wall geometry (packing
    // with the node barrier, then the device call), the box -> row maps
    std::snprintf(buf, sizeof buf,
                  ", \"upload_flatten\": %.6f, \"upload_lists\": %.6f, "
                  "\"upload_wall_pack\": %.6f, \"upload_wall_device\": %.6f, "
                  "\"upload_rows_map\": %.6f",
                  rg_up.flatten, rg_up.lists, rg_up.wall_pack, rg_up.wall_device, rg_up.rows_map);
    rphases += buf;
#endif
    rphases += "}";
  }
#ifdef ORACLE_BINDING
  {
    // moving-body phases on rank 0, all steps (warm-up included)
    const IbgpuMoveTimes &mt = ibgpu_move_times();
    char buf[768];
    std::snprintf(buf, sizeof buf,
                  "{\"forces\": %.6f, \"motion\": %.6f, \"distance\": %.6f, \"sync\": %.6f, "
                  "\"ibcells\": %.6f, \"upload\": %.6f, \"wall_pack\": %.6f, "
                  "\"wall_device\": %.6f, \"wall_unpack\": %.6f, \"ib_infect\": %.6f, "
                  "\"ib_compact\": %.6f, \"ib_image\": %.6f, \"ib_exchange\": %.6f, "
                  "\"ib_ghost\": %.6f, \"ib_patch\": %.6f, \"distcheck_mismatches\": %lld}",
                  mt.forces, mt.motion, mt.distance, mt.sync, mt.ibcells, mt.upload, mt.wall_pack,
                  mt.wall_device, mt.wall_unpack, mt.ib_infect, mt.ib_compact, mt.ib_image,
                  mt.ib_exchange, mt.ib_ghost, mt.ib_patch, ibgpu_wall_check_mismatches());
    phases = buf;
  }
#endif
  if (nrank == 0)
    std::printf("ORACLE_RESULT {\"steps\": %d, \"loop_seconds\": %.9f, \"cell_updates\": %lld, "
                "\"cell_updates_per_s\": %.6e, \"t\": %.17g, \"dt\": %.17g, "
                "\"move_seconds\": %.9f, \"regrid_seconds\": %.9f, \"ranks\": %d, "
                "\"move_phases_seconds\": %s, \"regrid_phases_seconds\": %s}\n",
                nsteps - timed_from, loop_time, cell_updates,
                loop_time > 0 ? (double)cell_updates / loop_time : 0.0, t, dt, move_time,
                regrid_time, nprocs, phases.c_str(), rphases.c_str());
  std::fflush(stdout);
  MPI_Finalize();
  return 0;
}
