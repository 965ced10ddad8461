// Reference-side binding of the B200 time step: the code a maintainer adds to
// the reference solver so that its main loop steps on the GPU through the C
// ABI of include/ibgpu.h, keeping the NS_Solver / Mesh / Body interface.
//
// Include after the reference's own headers (AMR.H, Body.H, Mesh.H,
// NS_Solver.H).  The adapter reads the reference's non-public pair lists,
// boundary values and immersed-boundary records; the reference grants that
// with one line in each of AMR, AMRLevel, Mesh, Meshlevel, BCValues and Body:
//     friend struct IbgpuAdapter;
//
// What it replaces (main.cpp:84-116): the three calls
//     amr.InterfaceExchange(); Body::IBConditions_Image(mesh, bodies);
//     flowsolver.TimeMarching(amr);
// become the single GpuNS_Solver::TimeMarching(amr), which runs the
// coarse/fine exchange (AMRInterface.cpp:3-35), the immersed-body ghost
// cells (Body.cpp:1361-1496), the domain ghosts and the multistage update
// (NS_Solver.H:657-702) on the device.  Upload() runs after InitFlow and
// after every AMR::PerformAdaptive; Download() fills m_data before output,
// host-side force evaluation or a regrid reads it.
//
// In the reference's shared-memory MPI mode (one node of several ranks, every
// mesh and body array in a shared window) rank 0 of the node's share_comm
// drives the device; every rank runs the reference's own host code (mesh
// generation, regrids, the moving bodies' re-immersion) over its share of
// the shared arrays, and the device rank's results (status, dt, forces) are
// broadcast to the node.  One node: the device context holds the whole mesh.
#pragma once

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "ibgpu.h"

// case constants the reference defines in its case file (not in a header)
extern const double Ma;
extern double p_ref, area_ref, shear_ref;

// The reference's mesh, pair lists, boundary ghosts and immersed-boundary
// records as the C ABI's canonical lists (positions, never array indices).
// The cell rows of the device lists: one row per box of the z = 0 plane of
// every level, normal cells and 2-D ghosts, in level order and each level's
// array order (the cell list of ibgpu_upload_topology and the state rows).
struct IbgpuRows {
  int64_t n = 0;
  int32_t *level = nullptr, *ix = nullptr, *iy = nullptr, *box = nullptr;
  uint8_t *flags = nullptr;  // IBGPU_CELL_*
  double *prim = nullptr;    // 7 per row: roe, u, v, w, p, T, e
};

struct IbgpuLists {
  // the cell rows (IbgpuRows) as vectors, for a single-process flattening
  std::vector<int32_t> level, ix, iy;
  std::vector<uint8_t> flags;  // IBGPU_CELL_*
  std::vector<double> prim;    // 7 per row: roe, u, v, w, p, T, e
  std::vector<int> box;        // the row's index in its level's box array
  std::vector<int32_t> res, pro;              // 11 per pair (ibgpu_cf_pairs)
  std::vector<int32_t> bc;                    // 7 per ghost (ibgpu_bc)
  std::vector<double> bc_nmv, facevar;        // 3 per ghost, 7 per face
  double backpressure = 0.0, inlet_flow_angle = 0.0;
  std::vector<int32_t> ib_cell, patch;        // 18 / 17 per row (ibgpu_ib)
  std::vector<double> ib_cellf, patchf, body_center;  // 16 / 19 / 3 per row
};

// Wall-clock seconds (MPI_Wtime on this rank) of the moving-body phases,
// accumulated over GpuNS_Solver::MoveBodies calls: device forces and their
// broadcast, motion (Motion_Rule, ModifyBoxtoPatch), wall distances
// (RenewLevelDistance), their synchronisation to block ghosts
// (SynNormal_BlockDistance), the immersed-boundary cells and image points
// (RemoveIBCells .. FindPatchHangingNode), and the device upload of the new
// flags and records (UploadImmersion).
struct IbgpuMoveTimes {
  double forces = 0.0, motion = 0.0, distance = 0.0, sync = 0.0, ibcells = 0.0, upload = 0.0;
  // the device wall distances' parts (within distance): packing this rank's
  // share, the device rank's call, unpacking
  double wall_pack = 0.0, wall_device = 0.0, wall_unpack = 0.0;
  // the immersed-boundary part's pieces (within ibcells): removed and newly
  // infected cells, the IB array's compaction and index, the image cells,
  // the wall cells' exchange, the ghost IB cells, the patches' hanging nodes
  double ib_infect = 0.0, ib_compact = 0.0, ib_image = 0.0, ib_exchange = 0.0, ib_ghost = 0.0,
         ib_patch = 0.0;
};
inline IbgpuMoveTimes &ibgpu_move_times() {
  static IbgpuMoveTimes t;
  return t;
}

// Seconds spent in GpuNS_Solver::Upload after regrids (this rank):
// flattening the mesh into the device lists (device rank), the lists'
// upload, and the wall geometry (windows, packing, the device call).
struct IbgpuUploadTimes {
  // wall_geometry = wall_pack (every rank's share, then the node barrier) +
  // wall_device (ibgpu_wall_geometry on the device rank, status shared)
  double flatten = 0.0, lists = 0.0, wall_geometry = 0.0, wall_pack = 0.0, wall_device = 0.0,
         rows_map = 0.0;
};
inline IbgpuUploadTimes &ibgpu_upload_times() {
  static IbgpuUploadTimes t;
  return t;
}

// The rank that drives the device: rank 0 of the node (share_comm,
// mpiparams.cpp:68-105).
inline bool ibgpu_device_rank() { return srank == 0; }
// An ibgpu status of the device rank, known to every rank of the node.
inline int ibgpu_share_status(int rc) {
  MPI_Bcast(&rc, 1, MPI_INT, 0, share_comm);
  return rc;
}

// A byte buffer shared by the ranks of the node: a shared window on
// share_comm, all of it held by rank 0 (collective allocation and release).
// With pin the device rank pins it for its transfers (ibgpu_host_register).
struct IbgpuSharedBytes {
  MPI_Win win;
  char *base = nullptr;
  size_t cap = 0;
  bool live = false, pinned = false;
  // at least nbytes: the buffer stays when it is large enough (a regrid
  // changes the box counts a little; a new window and its pinning cost far
  // more than the copies), else a new one with a quarter to spare
  void ensure(size_t nbytes, bool pin) {
    if (live && nbytes <= cap) return;  // the same decision on every rank (collective)
    alloc(nbytes + nbytes / 4, pin);
  }
  void alloc(size_t nbytes, bool pin) {
    release();
    cap = nbytes;
    char *local = nullptr;
    MPI_Win_allocate_shared(srank == 0 ? (MPI_Aint)nbytes : 0, 1, MPI_INFO_NULL, share_comm,
                            &local, &win);
    MPI_Aint sz;
    int du;
    MPI_Win_shared_query(win, 0, &sz, &du, &base);
    live = true;
    pinned = pin && srank == 0 && nbytes > 0 && ibgpu_host_register(base, nbytes) == IBGPU_OK;
  }
  void release() {
    if (pinned) ibgpu_host_unregister(base);
    if (live) MPI_Win_free(&win);
    live = pinned = false;
    base = nullptr;
    cap = 0;
  }
};

// One level's exchange buffers of the device wall distances
// (ibgpu_wall_geometry / ibgpu_wall_distance): every rank packs and unpacks
// its share of the boxes (DataArray::GlobalOrder) and of the block pairs
// (DataArray::ps/pe, the shares SynNormal_BlockDistance works on).
struct IbgpuWallLevel {
  int64_t n = 0, nblock = 0;
  IbgpuSharedBytes mem;
  double *center = nullptr, *dtdm = nullptr, *dist = nullptr, *sd = nullptr, *dtb = nullptr;
  int32_t *neib = nullptr, *body = nullptr, *patch = nullptr, *block_in = nullptr,
          *block_out = nullptr;
  uint8_t *kind = nullptr, *solid = nullptr, *moved = nullptr, *block_moved = nullptr;
  // the near-wall report of a move from the pairs the device kept
  // (ibgpu_wall_distance_near): its entries, in box order, and their number
  ibgpu_wall_change *changes = nullptr;
  int64_t *nchanges = nullptr;
  void layout(int64_t n_, int64_t nb_) {
    n = n_;
    nblock = nb_;
    size_t off = 0;
    auto take = [&off](size_t bytes) {
      const size_t o = off;
      off += (bytes + 15) & ~(size_t)15;
      return o;
    };
    const size_t oc = take(24 * n), odm = take(8 * n), odi = take(8 * n), osd = take(8 * n),
                 otb = take(8 * n), one = take(36 * n), obo = take(4 * n), opa = take(4 * n),
                 obi = take(4 * nblock), obu = take(4 * nblock), oki = take(n), oso = take(n),
                 omo = take(n), obm = take(nblock), och = take(sizeof(ibgpu_wall_change) * n),
                 onc = take(sizeof(int64_t));
    mem.ensure(off, true);
    char *b = mem.base;
    center = (double *)(b + oc);
    dtdm = (double *)(b + odm);
    dist = (double *)(b + odi);
    sd = (double *)(b + osd);
    dtb = (double *)(b + otb);
    neib = (int32_t *)(b + one);
    body = (int32_t *)(b + obo);
    patch = (int32_t *)(b + opa);
    block_in = (int32_t *)(b + obi);
    block_out = (int32_t *)(b + obu);
    kind = (uint8_t *)(b + oki);
    solid = (uint8_t *)(b + oso);
    moved = (uint8_t *)(b + omo);
    block_moved = (uint8_t *)(b + obm);
    changes = (ibgpu_wall_change *)(b + och);
    nchanges = (int64_t *)(b + onc);
  }
};

// Boxes whose device wall distances differed from the reference's own
// (GpuNS_Solver::SetWallDistanceCheck), summed over the node's ranks and
// every checked move.
inline long long &ibgpu_wall_check_mismatches() {
  static long long n = 0;
  return n;
}

struct IbgpuAdapter {
  // Case constants (gas constants, stage coefficients, levels, schedules,
  // domain, force scales) from the reference's globals and the solver's
  // stage scheme (NS_Solver.H:200-231).  The limiter is the reference's
  // compile-time ALimiter choice (Slopelimiter.H:20, 84-87).
  static ibgpu_case MakeCase(const NS_Solver &s, int limiter, int precision) {
    ibgpu_case c;
    std::memset(&c, 0, sizeof c);
    c.abi_version = IBGPU_ABI_VERSION;
    c.gama = gama;
    c.Rg = Rg;
    c.Cv = Cv;
    c.Cp = Cp;
    c.Ma = Ma;
    c.Re = Re;
    c.Pr = Pr;
    c.qk = qk;
    c.s_over_t = S_over_T_ref;
    c.cfl = CFL;
    c.dt_ratio = dt_ratio;
    c.dt_var_step = dt_var_step;
    c.nstages = s.sub_time_step;
    for (int k = 0; k < s.sub_time_step && k < 4; ++k) c.tp[k] = s.tp[k];
    c.limiter = limiter;
#ifdef VISCOUSITY
    c.viscous = 1;
#else
    c.viscous = 0;
#endif
    c.precision = precision;
    const double iv[7] = {initvar.roe, initvar.u, initvar.v, initvar.w,
                          initvar.p,   initvar.T, initvar.e};
    for (int k = 0; k < 7; ++k) c.initvar[k] = iv[k];
    const int nlev = s.a_mesh.MyCurNum();
    c.nlevels = nlev;
    for (int l = 0; l < nlev && l < IBGPU_MAX_LEVELS; ++l) {
      for (int k = 0; k < 3; ++k) c.dh[l][k] = dh[l][k];
      c.march_step[l] = marching_step[l];
      c.march_left[l] = marching_left_step[l];
      c.step_num[l] = step_num[l];
      c.average_step[l] = average_step[l];
      c.average_left[l] = average_left_step[l];
      c.prolong_step[l] = prolongation_step[l];
      c.prolong_left[l] = prolongation_left_step[l];
    }
    c.domain_nx = highpt.xy[0];
    c.domain_ny = highpt.xy[1];
    c.periodic_x = periodic[0] ? 1 : 0;
    c.periodic_y = periodic[1] ? 1 : 0;
    c.body_level = Body::Bodynum() > 0 ? nlev - 1 : -1;
    c.p_ref = p_ref;
    c.area_ref = area_ref;
    c.shear_ref = shear_ref;
    c.L_ref = L_ref;
    c.mu = mu;
    return c;
  }

  // The code path UpdateConsVars / ComptNewPrimVar / ResinDomain take for a
  // box (NS_Solver.cpp:3-194, 844-985; NS_Solver.H:264-378): on the finest
  // level of a run with bodies only non-solid boxes outside the immersed
  // boundary are updated, elsewhere every leaf box; a leaf box inside a body
  // (signed distance <= 0) is reset to the free stream.  Block (periodic)
  // ghosts are copies of the wrapped cell (Mesh::DataExchange).
  static uint8_t CellFlags(bool normal, bool block_ghost, bool solid, bool free_of_ib,
                           double signdis, bool body_level) {
    uint8_t f = IBGPU_CELL_PRESENT;
    if (normal) f |= IBGPU_CELL_NORMAL;
    const bool pos = signdis > 0.0;
    if (body_level) {
      const bool upd = normal && free_of_ib && !solid;
      if (upd) f |= IBGPU_CELL_UPDATE;
      if (upd && pos) f |= IBGPU_CELL_PRIM;
      if (normal && free_of_ib && !pos) f |= IBGPU_CELL_RESET;
      if (normal && free_of_ib && pos) f |= IBGPU_CELL_RESNORM;
    } else if (normal) {
      f |= IBGPU_CELL_UPDATE | IBGPU_CELL_RESNORM;
      f |= pos ? IBGPU_CELL_PRIM : IBGPU_CELL_RESET;
    }
    if (block_ghost) f |= IBGPU_CELL_ALIAS;
    return f;
  }

  static void Pos(std::vector<int32_t> &v, Mesh &mesh, int l, int b) {
    if (b < 0) {
      v.push_back(INT32_MIN);
      v.push_back(INT32_MIN);
      return;
    }
    Box &bx = mesh.ShowLevelBox(l)[b];
    v.push_back(bx.ix());
    v.push_back(bx.iy());
  }

  // IBGPU_CELL_* flags of box b of level l as the mesh holds it now.
  static uint8_t BoxFlags(Mesh &mesh, int l, int b) {
    const int nlev = mesh.MyCurNum();
    DataArray<Box> &boxes = mesh.ShowLevelBox(l);
    Box &bx = boxes[b];
    int infect = -1;
    if (l == nlev - 1 && mesh.Infectboxnum() > b) infect = mesh.BoxInfectIndex(b);
    const int nnorm = boxes.size();
    return CellFlags(b < nnorm, b >= nnorm && bx.type == Blockghost, bx.solid, infect == -1,
                     bx.pair.signdis, Body::Bodynum() > 0 && l == nlev - 1);
  }

  // Every list of the device from the mesh (one process).
  static void Flatten(Mesh &mesh, AMR &amr, std::vector<Body> &bodies, NS_Solver &solver,
                      IbgpuLists &L) {
    L = IbgpuLists();
    FlattenRows(mesh, L);
    FlattenLists(mesh, amr, bodies, solver, L);
  }

  static IbgpuRows RowsOf(IbgpuLists &L) {
    IbgpuRows R;
    R.n = (int64_t)L.level.size();
    R.level = L.level.data();
    R.ix = L.ix.data();
    R.iy = L.iy.data();
    R.box = L.box.data();
    R.flags = L.flags.data();
    R.prim = L.prim.data();
    return R;
  }

  // One cell row (IbgpuRows) of box b of level l.
  static void FillRow(Mesh &mesh, int l, int b, const IbgpuRows &R, int64_t i) {
    Box &bx = mesh.ShowLevelBox(l)[b];
    R.level[i] = l;
    R.ix[i] = bx.ix();
    R.iy[i] = bx.iy();
    R.box[i] = b;
    R.flags[i] = BoxFlags(mesh, l, b);
    FlowVariables &fv = mesh.LevelDataArray(l)[b];
    double *q = R.prim + 7 * i;
    q[0] = fv.roe;
    q[1] = fv.u;
    q[2] = fv.v;
    q[3] = fv.w;
    q[4] = fv.p;
    q[5] = fv.T;
    q[6] = fv.e;
  }

  // The cell rows: Meshlevel::m_box / m_data (Meshlevel.H:688-872).
  static void FlattenRows(Mesh &mesh, IbgpuLists &L) {
    const int nlev = mesh.MyCurNum();
    for (int l = 0; l < nlev; ++l) {
      DataArray<Box> &boxes = mesh.ShowLevelBox(l);
      DataArray<FlowVariables> &data = mesh.LevelDataArray(l);
      const int nreal = boxes.realsize();
      for (int b = 0; b < nreal; ++b) {
        Box &bx = boxes[b];
        if (bx.iz() != 0) continue;
        L.level.push_back(l);
        L.ix.push_back(bx.ix());
        L.iy.push_back(bx.iy());
        L.box.push_back(b);
        L.flags.push_back(BoxFlags(mesh, l, b));
        FlowVariables &fv = data[b];
        const double r[7] = {fv.roe, fv.u, fv.v, fv.w, fv.p, fv.T, fv.e};
        L.prim.insert(L.prim.end(), r, r + 7);
      }
    }
  }

  // The pair, domain-ghost and immersed-boundary lists.
  static void FlattenLists(Mesh &mesh, AMR &amr, std::vector<Body> &bodies, NS_Solver &solver,
                           IbgpuLists &L) {
    const int nlev = mesh.MyCurNum();
    // coarse/fine pairs: AMRLevel::f_res_ghost, f_pro_ghost, g_pro
    // (AMRLevel.H:320-329), the four z = 0 sons in Point_iterator_2d order
    for (int l = 0; l + 1 < nlev; ++l) {
      AMRLevel &al = amr.m_level[l];
      auto pair = [&](std::vector<int32_t> &v, CtoFPair &p) {
        v.push_back(l);
        Pos(v, mesh, l, p.ci);
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) Pos(v, mesh, l + 1, p.fi.son[a][b][0]);
      };
      for (int ig = 0; ig < ighost; ++ig)
        for (int i = 0; i < al.f_res_ghost[ig].size(); ++i) pair(L.res, al.f_res_ghost[ig][i]);
      for (int i = 0; i < al.f_pro_ghost.size(); ++i) pair(L.pro, al.f_pro_ghost[i]);
      for (int i = 0; i < al.g_pro.size(); ++i) pair(L.pro, al.level_pro_ghost[al.g_pro[i]]);
    }
    // domain ghosts of the x and y faces in BCBoxTreat order (BCValues.H:51-188)
    for (int l = 0; l < nlev; ++l) {
      DataArray<Domainghost> &dmg = mesh.MeshGhostArray(l);
      for (int i = 0; i < dmg.size(); ++i) {
        const int f0 = dmg[i].nbface;
        if (mesh.m_dm.facedir[f0][2] != 0 || mesh.ShowLevelBox(l)[dmg[i].cell].iz() != 0) continue;
        L.bc.push_back(l);
        Pos(L.bc, mesh, l, dmg[i].cell);
        Pos(L.bc, mesh, l, dmg[i].refcell);
        L.bc.push_back(f0);
        L.bc.push_back(mesh.m_dm.facetype[f0]);
        for (int k = 0; k < 3; ++k) L.bc_nmv.push_back(dmg[i].nmv[k]);
      }
    }
    BCValues &B = solver.meshbc;
    for (size_t f = 0; f < B.facevar.size(); ++f) {
      FlowVariables &v = B.facevar[f];
      const double r[7] = {v.roe, v.u, v.v, v.w, v.p, v.T, v.e};
      L.facevar.insert(L.facevar.end(), r, r + 7);
    }
    L.backpressure = B.backpressure;
    L.inlet_flow_angle = inlet_flow_angle;
    FlattenImmersed(mesh, bodies, L);
  }

  // The immersed-boundary cells and wall patches of the bodies where they
  // are now (replaces L's records of that kind).
  static void FlattenImmersed(Mesh &mesh, std::vector<Body> &bodies, IbgpuLists &L) {
    L.ib_cell.clear();
    L.ib_cellf.clear();
    L.patch.clear();
    L.patchf.clear();
    L.body_center.clear();
    const int nlev = mesh.MyCurNum();
    // immersed-boundary cells of the finest level (IBCell, Body.cpp:1361-1496)
    const int last = nlev - 1;
    DataArray<IBCell> &mdis = mesh.ibarray();
    for (int i = 0; i < mdis.size(); ++i) {
      IBCell &c = mdis[i];
      if (!(mesh.m_level[last].m_box.isnormal(c.ci) && c.mynode == node)) continue;
      BoxtoWall &w = mesh.m_level[last].m_box[c.ci].pair;
      Pos(L.ib_cell, mesh, last, c.ci);
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          for (int k = 0; k < 2; ++k) Pos(L.ib_cell, mesh, last, c.hgc.intpcell[a][b][k]);
      Pointxyz wall_v;
      bodies[w.body].Surface_Point_Velocity(c.hgc.attach_pt, wall_v);
      Pointxyz &nv = bodies[w.body].patch[w.patch].nv;
      L.ib_cellf.push_back(w.signdis);
      L.ib_cellf.push_back(c.hgc.hgdis);
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          for (int k = 0; k < 2; ++k) L.ib_cellf.push_back(c.hgc.intpcoef[a][b][k]);
      for (int k = 0; k < 3; ++k) L.ib_cellf.push_back(nv[k]);
      for (int k = 0; k < 3; ++k) L.ib_cellf.push_back(wall_v[k]);
    }
    // wall patches of Body::ComptWallForce (Body.cpp:439-558)
    for (size_t bi = 0; bi < bodies.size(); ++bi) {
      Body &Bd = bodies[bi];
      for (int k = 0; k < 3; ++k) L.body_center.push_back(Bd.bodycenter[k]);
      for (int i = 0; i < Bd.patch.size(); ++i) {
        Surfpatch &P = Bd.patch[i];
        if (P.node != node) continue;
        L.patch.push_back((int32_t)bi);
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b)
            for (int k = 0; k < 2; ++k) Pos(L.patch, mesh, last, P.hgc.intpcell[a][b][k]);
        for (int k = 0; k < 3; ++k) L.patchf.push_back(P.pc[k]);
        for (int k = 0; k < 3; ++k) L.patchf.push_back(P.nv[k]);
        L.patchf.push_back(P.area);
        L.patchf.push_back(P.hgc.hgdis);
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b)
            for (int k = 0; k < 2; ++k) L.patchf.push_back(P.hgc.intpcoef[a][b][k]);
        Pointxyz wall_v;
        Bd.Surface_Point_Velocity(P.pc, wall_v);
        for (int k = 0; k < 3; ++k) L.patchf.push_back(wall_v[k]);
      }
    }
  }

  // Boxes of the z = 0 plane in a level's range [ps, pe) as AMR::TagtheBox
  // judges them: position, centre (Mesh::bc) and signed wall distance.
  struct TagBoxes {
    std::vector<int32_t> level, ix, iy;
    std::vector<double> xc, yc, signdis;
    std::vector<int> box;  // index in the level's box array
  };
  static void GatherTagBoxes(Mesh &mesh, AMR &amr, int level, TagBoxes &T) {
    T = TagBoxes();
    AMRLevel &al = amr.m_level[level];
    for (int i = al.m_box.ps(); i < al.m_box.pe(); ++i) {
      Box &b = al.m_box[i];
      if (b.iz() != 0) continue;
      T.level.push_back(level);
      T.ix.push_back(b.ix());
      T.iy.push_back(b.iy());
      T.xc.push_back(mesh.bc(level, i)[0]);
      T.yc.push_back(mesh.bc(level, i)[1]);
      T.signdis.push_back(b.pair.signdis);
      T.box.push_back(i);
    }
  }

  // The case's regions with the requests of this regrid for `level`: the
  // reference's AMR::TagtheBox acts only when the level's own
  // AMRLevel::torefine / toderefine are set (Userfunction_cy_naca15.cpp:557,
  // 590), and ADPRule / SetRefineFlag set them level by level, so a rule
  // built once for the case never decides the request itself.
  static ibgpu_tag_rule LevelRule(const ibgpu_tag_rule &rule, AMR &amr, int level) {
    ibgpu_tag_rule r = rule;
    if (level >= 0 && level < IBGPU_TAG_MAX_LEVELS) {
      r.torefine[level] = amr.m_level[level].torefine ? 1 : 0;
      r.toderefine[level] = amr.m_level[level].toderefine ? 1 : 0;
    }
    return r;
  }

  // Decisions (IBGPU_TAG_* bits of the boxes T) into m_tag / taggedbox, as
  // the tagging loops leave them.
  static void ApplyTags(AMR &amr, int level, const TagBoxes &T, const std::vector<uint8_t> &bits) {
    AMRLevel &al = amr.m_level[level];
    for (size_t k = 0; k < bits.size(); ++k) {
      const int i = T.box[k];
      if (bits[k] & IBGPU_TAG_REFINE) {
        al.m_tag[i].givetag();
        al.taggedbox.push_back(i);
      }
      if (bits[k] & IBGPU_TAG_COARSEN) al.m_tag[i].givedetag();
    }
  }

  // The tagging loops of a case's AMR::TagtheBox (Userfunction_cy_naca15.cpp
  // :560-635) for one level through the C ABI: the plain criterion
  // (ibgpu_tag_plain) or, with device MLP parameters, the learned indicator
  // (ibgpu_tag_learned, reading the context's uploaded state), with the
  // level's own refine / coarsen requests (LevelRule); the decisions land in
  // m_tag / taggedbox as the loops leave them.  Call after Inittag();
  // CheckDetagLocation stays the caller's.
  static int TagLevel(ibgpu_ctx *ctx, const ibgpu_tag_rule &rule, Mesh &mesh, AMR &amr,
                      int level, const float *d_params) {
    TagBoxes T;
    GatherTagBoxes(mesh, amr, level, T);
    const ibgpu_tag_rule lr = LevelRule(rule, amr, level);
    const ibgpu_tag_cells q = {(int64_t)T.box.size(), T.level.data(), T.ix.data(), T.iy.data(),
                               T.xc.data(), T.yc.data(), T.signdis.data()};
    std::vector<uint8_t> bits(T.box.size());
    const int rc = d_params ? ibgpu_tag_learned(ctx, &lr, &q, d_params, bits.data())
                            : ibgpu_tag_plain(ctx, &lr, &q, bits.data());
    if (rc) return rc;
    ApplyTags(amr, level, T, bits);
    return IBGPU_OK;
  }

  // ---- device wall distances (every rank of the node calls these)

  // After a regrid: every level's boxes (centres, in-plane neighbours,
  // kinds, distances to the domain boundary) and block pairs into the
  // levels' exchange buffers and the device.
  static int WallGeometry(ibgpu_ctx *ctx, Mesh &mesh, std::vector<IbgpuWallLevel> &W) {
    const double t0 = MPI_Wtime();
    const int nlev = mesh.MyCurNum();
    // the levels' windows stay from the last regrid where they are large
    // enough (every rank computes the same sizes, so all keep or renew alike)
    for (size_t l = (size_t)nlev; l < W.size(); ++l) W[l].mem.release();
    W.resize(nlev);
    for (int l = 0; l < nlev; ++l) {
      DataArray<Box> &boxes = mesh.ShowLevelBox(l);
      DataArray<NodePair> &bp = mesh.m_level[l].blockpair;
      IbgpuWallLevel &L = W[l];
      L.layout(boxes.realsize(), bp.size());
      int bs, be;
      boxes.GlobalOrder(bs, be);
      for (int i = bs; i < be; ++i) {
        Box &bx = boxes[i];
        Pointxyz &c = mesh.m_level[l].m_geom[i].boxcenter;
        for (int k = 0; k < 3; ++k) L.center[3 * i + k] = c[k];
        L.dtdm[i] = bx.pair.distance_to_dm;
        L.kind[i] = bx.type == Dmghost ? IBGPU_WALL_BOX_DOMAIN_GHOST
                    : bx.type == Blockghost ? IBGPU_WALL_BOX_BLOCK_GHOST
                                            : IBGPU_WALL_BOX_OTHER;
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) L.neib[9 * i + 3 * a + b] = bx.neib[a][b][1];
      }
      for (int k = bp.ps(); k < bp.pe(); ++k) {
        L.block_in[k] = bp[k].innode;
        L.block_out[k] = bp[k].outnode.index;
      }
    }
    MPI_Barrier(share_comm);
    IbgpuUploadTimes &tu = ibgpu_upload_times();
    const double t1 = MPI_Wtime();
    tu.wall_pack += t1 - t0;
    int rc = IBGPU_OK;
    if (ibgpu_device_rank()) {
      std::vector<ibgpu_wall_level_geom> g(nlev);
      for (int l = 0; l < nlev; ++l) {
        IbgpuWallLevel &L = W[l];
        g[l] = ibgpu_wall_level_geom{L.n, L.center, L.neib, L.kind, L.dtdm, L.nblock,
                                     L.block_in, L.block_out};
      }
      rc = ibgpu_wall_geometry(ctx, nlev, g.data());
    }
    rc = ibgpu_share_status(rc);
    tu.wall_device += MPI_Wtime() - t1;
    return rc;
  }

  // The wall distances of the moved bodies on the device: every level's
  // pairs as they are, computed anew (Body::RenewLevelDistance of every
  // level, then Mesh::SynNormal_BlockDistance's block-ghost copies).  With
  // apply the boxes take the new pairs and solid flags and this rank's move
  // lists get the boxes of its shares that changed sides, in the order the
  // reference's loops would push them; without, the results stay in W.
  // With resident the device starts from the pairs it kept from its
  // previous call (nothing but these passes changes the pairs between
  // regrids) and no rank packs; applied, it then reports only the boxes
  // near a wall before or after the move or on the other side now
  // (ibgpu_wall_distance_near, kWallNearCells cells of each level), the
  // boxes the reference's re-immersion reads before the next move.
  static int WallDistances(ibgpu_ctx *ctx, Mesh &amesh, std::vector<Body> &abody,
                           std::vector<IbgpuWallLevel> &W, bool apply, bool resident,
                           std::vector<std::vector<int> > &in_to_out,
                           std::vector<std::vector<int> > &out_to_in) {
    const int nlev = amesh.MyCurNum();
    if ((int)W.size() != nlev) return IBGPU_E_STATE;
    IbgpuMoveTimes &tm = ibgpu_move_times();
    double t0 = MPI_Wtime();
    for (int l = 0; l < nlev && !resident; ++l) {
      DataArray<Box> &boxes = amesh.ShowLevelBox(l);
      IbgpuWallLevel &L = W[l];
      int bs, be;
      boxes.GlobalOrder(bs, be);
      for (int i = bs; i < be; ++i) {
        const BoxtoWall &w = boxes[i].pair;
        L.body[i] = w.body;
        L.patch[i] = w.patch;
        L.dist[i] = w.distance;
        L.sd[i] = w.signdis;
        L.dtb[i] = w.distance_to_body;
        L.solid[i] = boxes[i].solid ? 1 : 0;
      }
    }
    MPI_Barrier(share_comm);
    double t1 = MPI_Wtime();
    tm.wall_pack += t1 - t0;
    t0 = t1;
    int rc = IBGPU_OK;
    if (ibgpu_device_rank()) {
      // the bodies' wall patches where they are now (small: the device rank alone)
      const int nb = (int)abody.size();
      std::vector<int32_t> start(nb + 1, 0), nbc, nbl;
      std::vector<double> pc, nv;
      for (int b = 0; b < nb && rc == IBGPU_OK; ++b) {
        Body &B = abody[b];
        if (B.bodyindex != b) rc = IBGPU_E_ARG;
        const int np = B.patch.size();
        start[b + 1] = start[b] + np;
        for (int p = 0; p < np; ++p) {
          for (int k = 0; k < 3; ++k) pc.push_back(B.patch[p].pc[k]);
          for (int k = 0; k < 3; ++k) nv.push_back(B.patch[p].nv[k]);
          nbc.push_back(B.patneib[p].nbnum);
          for (int k = 0; k < IBGPU_WALL_MAX_NB; ++k)
            nbl.push_back(k < B.patneib[p].nbnum ? B.patneib[p].nb[k] : -1);
        }
      }
      if (rc == IBGPU_OK) {
        const ibgpu_wall_bodies wb = {nb, start.data(), pc.data(), nv.data(), nbc.data(),
                                      nbl.data(), periodic[1] ? 1 : 0, critic_ylength,
                                      dmlength[1]};
        if (resident && apply) {
          std::vector<ibgpu_wall_near> near(nlev);
          for (int l = 0; l < nlev; ++l) {
            IbgpuWallLevel &L = W[l];
            near[l] = ibgpu_wall_near{kWallNearCells * dh[l][0], L.n, L.changes, 0,
                                      L.block_moved};
          }
          rc = ibgpu_wall_distance_near(ctx, &wb, nlev, near.data());
          for (int l = 0; l < nlev; ++l) *W[l].nchanges = near[l].count;
        } else {
          std::vector<ibgpu_wall_pairs> pr(nlev);
          for (int l = 0; l < nlev; ++l) {
            IbgpuWallLevel &L = W[l];
            pr[l] = ibgpu_wall_pairs{L.body, L.patch, L.dist, L.sd, L.dtb, L.solid, L.moved,
                                     L.block_moved};
          }
          rc = ibgpu_wall_distance(ctx, &wb, nlev, pr.data(), resident ? IBGPU_WALL_RESIDENT : 0);
        }
      }
    }
    rc = ibgpu_share_status(rc);
    MPI_Barrier(share_comm);
    t1 = MPI_Wtime();
    tm.wall_device += t1 - t0;
    t0 = t1;
    if (rc != IBGPU_OK || !apply) return rc;
    if (resident) WallUnpackNear(amesh, W, in_to_out, out_to_in);
    else WallUnpack(amesh, W, true, &in_to_out, &out_to_in);
    tm.wall_unpack += MPI_Wtime() - t0;
    return IBGPU_OK;
  }

  // The near-wall report of the last move into this rank's shares of the
  // boxes (the report is in box order, so a share is one run of it), with
  // this rank's move-list entries in the order the reference's loops push
  // them; the other boxes keep their previous pairs on the host until
  // Download fetches every pair.
  static void WallUnpackNear(Mesh &amesh, std::vector<IbgpuWallLevel> &W,
                             std::vector<std::vector<int> > &in_to_out,
                             std::vector<std::vector<int> > &out_to_in) {
    for (size_t l = 0; l < W.size(); ++l) {
      DataArray<Box> &boxes = amesh.ShowLevelBox((int)l);
      DataArray<NodePair> &bp = amesh.m_level[l].blockpair;
      IbgpuWallLevel &L = W[l];
      int bs, be;
      boxes.GlobalOrder(bs, be);
      const ibgpu_wall_change *c = L.changes, *end = L.changes + *L.nchanges;
      c = std::lower_bound(c, end, bs,
                           [](const ibgpu_wall_change &a, int box) { return a.box < box; });
      for (; c != end && c->box < be; ++c) {
        const int i = c->box;
        BoxtoWall &w = boxes[i].pair;
        w.body = c->body;
        w.patch = c->patch;
        w.distance = c->distance;
        w.signdis = c->signdis;
        w.distance_to_body = c->distance_to_body;
        boxes[i].solid = c->solid != 0;
        if (c->moved == IBGPU_WALL_INTO_BODY) out_to_in[l].push_back(i);
        else if (c->moved == IBGPU_WALL_OUT_OF_BODY) in_to_out[l].push_back(i);
      }
      for (int k = bp.ps(); k < bp.pe(); ++k) {
        if (L.block_moved[k] == IBGPU_WALL_INTO_BODY) out_to_in[l].push_back(L.block_out[k]);
        else if (L.block_moved[k] == IBGPU_WALL_OUT_OF_BODY)
          in_to_out[l].push_back(L.block_out[k]);
      }
    }
    MPI_Barrier(share_comm);  // every box written before the reference's next loops
  }

  // The device's last wall-distance results (in W) into this rank's shares
  // of the boxes.  With near only the boxes the re-immersion reads before
  // the next move: within kWallNearCells cells of the level from a wall,
  // or that changed sides; the others keep their previous pairs on the host
  // (the device keeps them all) until a call without near, which Download
  // makes before any output or regrid reads the mesh.  With move lists this
  // rank's entries, in the order the reference's loops push them.
  static constexpr double kWallNearCells = 10.0;
  static void WallUnpack(Mesh &amesh, std::vector<IbgpuWallLevel> &W, bool near,
                         std::vector<std::vector<int> > *in_to_out,
                         std::vector<std::vector<int> > *out_to_in) {
    for (size_t l = 0; l < W.size(); ++l) {
      DataArray<Box> &boxes = amesh.ShowLevelBox((int)l);
      DataArray<NodePair> &bp = amesh.m_level[l].blockpair;
      IbgpuWallLevel &L = W[l];
      const double band = near ? kWallNearCells * dh[l][0] : HUGE_VAL;
      int bs, be;
      boxes.GlobalOrder(bs, be);
      for (int i = bs; i < be; ++i) {
        if (!(std::fabs(L.sd[i]) < band) && L.moved[i] == 0) continue;
        BoxtoWall &w = boxes[i].pair;
        w.body = L.body[i];
        w.patch = L.patch[i];
        w.distance = L.dist[i];
        w.signdis = L.sd[i];
        w.distance_to_body = L.dtb[i];
        boxes[i].solid = L.solid[i] != 0;
        if (!in_to_out) continue;
        if (L.moved[i] == IBGPU_WALL_INTO_BODY) (*out_to_in)[l].push_back(i);
        else if (L.moved[i] == IBGPU_WALL_OUT_OF_BODY) (*in_to_out)[l].push_back(i);
      }
      if (!in_to_out) continue;
      for (int k = bp.ps(); k < bp.pe(); ++k) {
        if (L.block_moved[k] == IBGPU_WALL_INTO_BODY) (*out_to_in)[l].push_back(L.block_out[k]);
        else if (L.block_moved[k] == IBGPU_WALL_OUT_OF_BODY)
          (*in_to_out)[l].push_back(L.block_out[k]);
      }
    }
    MPI_Barrier(share_comm);  // every box written before the reference's next loops
  }

  // Boxes of this rank's shares whose pair, solid flag or move-list entries
  // differ between the device results in W and the mesh as the reference's
  // own loops left it.
  static long long WallMismatches(Mesh &amesh, std::vector<IbgpuWallLevel> &W,
                                  const std::vector<std::vector<int> > &in_to_out,
                                  const std::vector<std::vector<int> > &out_to_in) {
    long long bad = 0;
    for (size_t l = 0; l < W.size(); ++l) {
      DataArray<Box> &boxes = amesh.ShowLevelBox((int)l);
      DataArray<NodePair> &bp = amesh.m_level[l].blockpair;
      IbgpuWallLevel &L = W[l];
      int bs, be;
      boxes.GlobalOrder(bs, be);
      std::vector<int> dev_in, dev_out;
      for (int i = bs; i < be; ++i) {
        const BoxtoWall &w = boxes[i].pair;
        if (w.body != L.body[i] || w.patch != L.patch[i] ||
            std::memcmp(&w.distance, &L.dist[i], 8) || std::memcmp(&w.signdis, &L.sd[i], 8) ||
            std::memcmp(&w.distance_to_body, &L.dtb[i], 8) || boxes[i].solid != (L.solid[i] != 0))
          ++bad;
        if (L.moved[i] == IBGPU_WALL_INTO_BODY) dev_in.push_back(i);
        else if (L.moved[i] == IBGPU_WALL_OUT_OF_BODY) dev_out.push_back(i);
      }
      for (int k = bp.ps(); k < bp.pe(); ++k) {
        if (L.block_moved[k] == IBGPU_WALL_INTO_BODY) dev_in.push_back(L.block_out[k]);
        else if (L.block_moved[k] == IBGPU_WALL_OUT_OF_BODY) dev_out.push_back(L.block_out[k]);
      }
      if (dev_in != out_to_in[l]) ++bad;
      if (dev_out != in_to_out[l]) ++bad;
    }
    return bad;
  }

  // Body::MovingBody_Image (Bodymove.cpp:37-125) for a run whose state lives
  // on the device: the bodies' forces and moments come from the device
  // (ibgpu_wall_forces, the wall patches as the last upload left them: the
  // reference's Body::ComptWallForce of the same patches), paired over the
  // two surfaces of each profile as the reference pairs them; then the
  // reference's own motion rule and re-immersion (wall distances of every
  // level, removed and newly infected immersed-boundary cells, image points),
  // and the patches' image-point stencils at the new position
  // (Body::FindPatchHangingNode, which the reference's next ComptWallForce
  // would run first).  The caller then hands the device the new flags and
  // records (GpuNS_Solver::UploadImmersion).
  // Every rank of the node calls it (the re-immersion is the reference's
  // own collective code); ctx is the device rank's context.
  // With W (the device wall distances, after WallGeometry) the distance
  // and block-ghost passes run on the device; with check also the
  // reference's own, the difference counted (ibgpu_wall_check_mismatches).
  static int MoveBodies(ibgpu_ctx *ctx, Mesh &amesh, std::vector<Body> &abody, double &dt00,
                        std::vector<IbgpuWallLevel> *W = nullptr, bool check = false,
                        bool *resident = nullptr) {
    const int nlev = amesh.MyCurNum();
    const int last = nlev - 1;
    std::vector<std::vector<int> > in_to_out(nlev), out_to_in(nlev);
    gridisnew = true;
    const int bn = (int)abody.size();
    IbgpuMoveTimes &tm = ibgpu_move_times();
    double t0 = MPI_Wtime();
    std::vector<double> fm(6 * (size_t)bn);
    if (bn > 0) {
      const int rc = ibgpu_share_status(ibgpu_device_rank() ? ibgpu_wall_forces(ctx, fm.data())
                                                            : IBGPU_OK);
      if (rc) return rc;
      MPI_Bcast(fm.data(), 6 * bn, MPI_DOUBLE, 0, share_comm);
    }
    for (int i = 0; i < bn; ++i)
      for (int k = 0; k < 3; ++k) {
        abody[i].draglift(k) = fm[6 * i + k];
        abody[i].bodymoment(k) = fm[6 * i + 3 + k];
      }
    for (int i = 0; i < bn / 2; ++i)
      for (int k = 0; k < 3; ++k) {
        abody[2 * i].draglift(k) += abody[2 * i + 1].draglift(k);
        abody[2 * i + 1].draglift(k) = abody[2 * i].draglift(k);
        abody[2 * i].bodymoment(k) += abody[2 * i + 1].bodymoment(k);
        abody[2 * i + 1].bodymoment(k) = abody[2 * i].bodymoment(k);
      }
    double t1 = MPI_Wtime();
    tm.forces += t1 - t0;
    t0 = t1;
    for (int i = 0; i < bn; ++i) {
      abody[i].Motion_Rule(amesh, dt00);
      abody[i].ModifyBoxtoPatch(amesh);
    }
    t1 = MPI_Wtime();
    tm.motion += t1 - t0;
    t0 = t1;
    if (W && !check) {
      const bool res = resident && *resident;
      const int rc = WallDistances(ctx, amesh, abody, *W, true, res, in_to_out, out_to_in);
      if (resident) *resident = rc == IBGPU_OK;
      if (rc) return rc;
      t1 = MPI_Wtime();
      tm.distance += t1 - t0;
      t0 = t1;
    } else {
      if (W) {  // the device's results first, from the same pairs
        const int rc = WallDistances(ctx, amesh, abody, *W, false, false, in_to_out, out_to_in);
        if (rc) return rc;
      }
      for (int l = 0; l < nlev; ++l) Body::RenewLevelDistance(amesh, abody, l, in_to_out[l], out_to_in[l]);
      t1 = MPI_Wtime();
      tm.distance += t1 - t0;
      t0 = t1;
      for (int l = 0; l < nlev; ++l) amesh.SynNormal_BlockDistance(l, in_to_out[l], out_to_in[l]);
      t1 = MPI_Wtime();
      tm.sync += t1 - t0;
      t0 = t1;
      if (W) {
        long long bad = WallMismatches(amesh, *W, in_to_out, out_to_in);
        MPI_Allreduce(MPI_IN_PLACE, &bad, 1, MPI_LONG, MPI_SUM, share_comm);
        ibgpu_wall_check_mismatches() += bad;
      }
    }
    double ti = MPI_Wtime();
    auto lap = [&ti](double &acc) {
      const double t = MPI_Wtime();
      acc += t - ti;
      ti = t;
    };
    Body::RemoveIBCells(amesh, abody, in_to_out[last], out_to_in[last]);
    Body::InfectNewIBCells(amesh, abody, in_to_out[last], out_to_in[last]);
    lap(tm.ib_infect);
    amesh.m_dis.holeplan(true);
    amesh.m_dis.CompressArray();
    amesh.RenewInfectIndex();
    lap(tm.ib_compact);
    Body::FindImageCell(amesh, abody);
    lap(tm.ib_image);
    amesh.DataExchangeCells_Wall();
    lap(tm.ib_exchange);
    Body::FindImageCell_GhostIBCell(amesh, abody);
    lap(tm.ib_ghost);
    for (int i = 0; i < bn; ++i) abody[i].FindPatchHangingNode(amesh);
    lap(tm.ib_patch);
    tm.ibcells += MPI_Wtime() - t0;
    return IBGPU_OK;
  }

  // The lists and the state into a context (ibgpu_upload_*).
  static int Upload(ibgpu_ctx *ctx, const IbgpuLists &L, const IbgpuRows &R) {
    ibgpu_cells cells = {R.n, R.level, R.ix, R.iy, R.flags};
    int rc = ibgpu_upload_topology(ctx, &cells);
    if (rc) return rc;
    ibgpu_cf_pairs cf = {(int64_t)L.res.size() / 11, L.res.data(), (int64_t)L.pro.size() / 11,
                         L.pro.data()};
    if ((rc = ibgpu_upload_interfaces(ctx, &cf))) return rc;
    ibgpu_bc bc = {(int64_t)L.bc.size() / 7, L.bc.data(), L.bc_nmv.data(),
                   (int)(L.facevar.size() / 7), L.facevar.data(), L.backpressure,
                   L.inlet_flow_angle};
    if ((rc = ibgpu_upload_boundaries(ctx, &bc))) return rc;
    if ((rc = UploadIB(ctx, L))) return rc;
    return ibgpu_upload_state(ctx, R.prim);
  }

  static int UploadIB(ibgpu_ctx *ctx, const IbgpuLists &L) {
    ibgpu_ib ib = {(int64_t)L.ib_cell.size() / 18, L.ib_cell.data(), L.ib_cellf.data(),
                   (int64_t)L.patch.size() / 17, L.patch.data(), L.patchf.data(),
                   (int)(L.body_center.size() / 3), L.body_center.data()};
    return ibgpu_upload_ib(ctx, &ib);
  }
};

// NS_Solver whose TimeMarching runs on the GPU.  TimeMarching is non-virtual
// and inline in the reference (NS_Solver.H:657-702), so the main loop holds
// the solver with this static type.
class GpuNS_Solver : public NS_Solver {
 public:
  GpuNS_Solver(Mesh &m, Domain &d, int nbody) : NS_Solver(m, d, nbody) {}
  GpuNS_Solver(const GpuNS_Solver &) = delete;
  GpuNS_Solver &operator=(const GpuNS_Solver &) = delete;
  ~GpuNS_Solver() {
    if (ctx_) ibgpu_destroy(ctx_);
  }

  // Device context for this case (IBGPU_FP64 / IBGPU_FP64_EXACT /
  // IBGPU_MIXED; the limiter as the reference was compiled with).  Every
  // rank of the node calls it; the device rank creates the context.
  int Create(int limiter, int precision) {
    if (created_) return IBGPU_E_STATE;
    int rc = IBGPU_OK;
    if (ibgpu_device_rank()) {
      const ibgpu_case c = IbgpuAdapter::MakeCase(*this, limiter, precision);
      rc = ibgpu_create(&c, &ctx_);
    }
    rc = ibgpu_share_status(rc);
    created_ = rc == IBGPU_OK;
    return rc;
  }

  // After InitFlow and after every AMR::PerformAdaptive (every rank).
  int Upload(AMR &amr, std::vector<Body> &bodies) {
    if (!created_) return IBGPU_E_STATE;
    MPI_Barrier(share_comm);  // every rank's share of the arrays written
    IbgpuUploadTimes &tu = ibgpu_upload_times();
    double t0 = MPI_Wtime();
    FlattenRowsShared();
    int rc = IBGPU_OK;
    if (ibgpu_device_rank()) {
      lists_ = IbgpuLists();
      IbgpuAdapter::FlattenLists(a_mesh, amr, bodies, *this, lists_);
      const double t1 = MPI_Wtime();
      tu.flatten += t1 - t0;
      t0 = t1;
      rc = IbgpuAdapter::Upload(ctx_, lists_, rows_);
    }
    rc = ibgpu_share_status(rc);
    tu.lists += MPI_Wtime() - t0;
    t0 = MPI_Wtime();
    if (rc == IBGPU_OK && device_distance_ && Body::Bodynum() > 0) {
      rc = IbgpuAdapter::WallGeometry(ctx_, a_mesh, wall_);
      wall_resident_ = false;  // the regrid's own pairs go up with the next move
    }
    tu.wall_geometry += MPI_Wtime() - t0;
    t0 = MPI_Wtime();
    if (rc == IBGPU_OK) {
      // each level's box -> row map (every rank, from the shared rows), for
      // the flag updates of the rows near the walls after a move
      row_of_.assign(a_mesh.MyCurNum(), std::vector<int>());
      for (int l = 0; l < a_mesh.MyCurNum(); ++l)
        row_of_[l].assign(a_mesh.ShowLevelBox(l).realsize(), -1);
      for (int64_t i = 0; i < rows_.n; ++i) row_of_[rows_.level[i]][rows_.box[i]] = (int)i;
      ib_rows_.clear();
    }
    tu.rows_map += MPI_Wtime() - t0;
    return rc;
  }

  // The cell rows (IbgpuRows) in a window shared by the node, every rank
  // filling the rows of its share of each level's boxes (collective; the
  // window stays across regrids while it is large enough, pinned on the
  // device rank for the state's transfers).
  void FlattenRowsShared() {
    const int nlev = a_mesh.MyCurNum();
    // this rank's boxes of each level and its rows among them
    std::vector<int> mine(nlev, 0), lo(nlev), hi(nlev);
    for (int l = 0; l < nlev; ++l) {
      DataArray<Box> &boxes = a_mesh.ShowLevelBox(l);
      const int64_t nreal = boxes.realsize();
      lo[l] = (int)(nreal * srank / sprocs);
      hi[l] = (int)(nreal * (srank + 1) / sprocs);
      for (int b = lo[l]; b < hi[l]; ++b) mine[l] += boxes[b].iz() == 0;
    }
    std::vector<int> all((size_t)nlev * sprocs);
    MPI_Allgather(mine.data(), nlev, MPI_INT, all.data(), nlev, MPI_INT, share_comm);
    // rows in level order, then rank order (each rank's share is a run of
    // its level's boxes), so in each level's array order: this rank's first
    // row of level l follows the rows of the levels before and of the ranks
    // before it
    std::vector<int64_t> off(nlev);
    int64_t n = 0;
    for (int l = 0; l < nlev; ++l)
      for (int r = 0; r < sprocs; ++r) {
        if (r == srank) off[l] = n;
        n += all[(size_t)r * nlev + l];
      }
    const size_t bytes = (size_t)n * (4 * sizeof(int32_t) + 1 + 7 * sizeof(double)) + 64;
    rows_mem_.ensure(bytes, true);
    char *base = rows_mem_.base;
    rows_.n = n;
    rows_.prim = (double *)base;  // 8-byte aligned first
    rows_.level = (int32_t *)(base + (size_t)n * 7 * sizeof(double));
    rows_.ix = rows_.level + n;
    rows_.iy = rows_.ix + n;
    rows_.box = rows_.iy + n;
    rows_.flags = (uint8_t *)(rows_.box + n);
    for (int l = 0; l < nlev; ++l) {
      DataArray<Box> &boxes = a_mesh.ShowLevelBox(l);
      int64_t i = off[l];
      for (int b = lo[l]; b < hi[l]; ++b)
        if (boxes[b].iz() == 0) IbgpuAdapter::FillRow(a_mesh, l, b, rows_, i++);
    }
    MPI_Barrier(share_comm);  // every rank's rows written
  }

  // The moving-body part of Body::IBConditions_Image (Body.cpp:1352-1357)
  // for a run stepping on the device: call before TimeMarching each step
  // when the case moves its bodies (moveflag), on every rank.  It
  // accumulates dt00 as the reference does, moves and re-immerses the
  // bodies on the host (IbgpuAdapter::MoveBodies) and hands the device the
  // new cell flags and immersed-boundary records; the state stays on the
  // device.
  int MoveBodies(std::vector<Body> &bodies, double &dt00) {
    if (!created_) return IBGPU_E_STATE;
    dt00 += dt;
    // a move from the pairs the device kept reports the boxes near the
    // walls, and only their rows' flags can change
    const bool near = device_distance_ && !wall_check_ && wall_resident_;
    int rc = IbgpuAdapter::MoveBodies(ctx_, a_mesh, bodies, dt00,
                                      device_distance_ ? &wall_ : nullptr, wall_check_,
                                      &wall_resident_);
    if (rc) return rc;
    dt00 = 0.0;
    const double t0 = MPI_Wtime();
    rc = UploadImmersion(bodies, near);
    ibgpu_move_times().upload += MPI_Wtime() - t0;
    return rc;
  }

  // Wall distances of moving bodies on the device (ibgpu_wall_distance) in
  // place of the reference's RenewLevelDistance and SynNormal_BlockDistance
  // (the default); with check, both, the reference's results kept and the
  // boxes that differ counted in ibgpu_wall_check_mismatches().  Set
  // before Upload, on every rank.
  void SetDeviceWallDistances(bool on, bool check = false) {
    device_distance_ = on;
    wall_check_ = on && check;
  }

  // After the bodies moved without a regrid: the flags of the same cell rows
  // (ibgpu_update_flags) and the immersed-boundary records
  // (ibgpu_upload_ib) from the mesh as it is now (every rank).  With near
  // (the move's wall distances came as the device's near-wall report) only
  // the rows whose flags the move can change: the reported boxes' rows
  // (each rank its run of every level's report) and the immersed-boundary
  // cells' rows before and after the move (ibgpu_update_flags_rows).
  int UploadImmersion(std::vector<Body> &bodies, bool near = false) {
    if (!created_) return IBGPU_E_STATE;
    MPI_Barrier(share_comm);
    if (near) return UploadImmersionNear(bodies);
    // the rows' flags into the shared rows, each rank a contiguous share
    const int64_t nrows = rows_.n;
    for (int64_t i = nrows * srank / sprocs; i < nrows * (srank + 1) / sprocs; ++i)
      rows_.flags[i] = IbgpuAdapter::BoxFlags(a_mesh, rows_.level[i], rows_.box[i]);
    MPI_Barrier(share_comm);
    int rc = IBGPU_OK;
    if (ibgpu_device_rank()) {
      // the immersed-boundary cells' rows, for the next update of the rows
      // near the walls
      const int last = a_mesh.MyCurNum() - 1;
      ib_rows_.clear();
      DataArray<IBCell> &mdis = a_mesh.ibarray();
      for (int i = 0; i < mdis.size(); ++i) {
        const int b = mdis[i].ci;
        if (b >= 0 && b < (int)row_of_[last].size() && row_of_[last][b] >= 0)
          ib_rows_.push_back(row_of_[last][b]);
      }
      rc = ibgpu_update_flags(ctx_, rows_.flags);
      if (rc == IBGPU_OK) {
        IbgpuAdapter::FlattenImmersed(a_mesh, bodies, lists_);
        rc = IbgpuAdapter::UploadIB(ctx_, lists_);
      }
    }
    return ibgpu_share_status(rc);
  }

  int UploadImmersionNear(std::vector<Body> &bodies) {
    const int nlev = a_mesh.MyCurNum();
    std::vector<int> rows;
    for (int l = 0; l < nlev && l < (int)wall_.size(); ++l) {
      DataArray<Box> &boxes = a_mesh.ShowLevelBox(l);
      const IbgpuWallLevel &W = wall_[l];
      const std::vector<int> &m = row_of_[l];
      int bs, be;
      boxes.GlobalOrder(bs, be);
      const ibgpu_wall_change *c = W.changes, *end = W.changes + *W.nchanges;
      c = std::lower_bound(c, end, bs,
                           [](const ibgpu_wall_change &a, int box) { return a.box < box; });
      for (; c != end && c->box < be; ++c)
        if (c->box < (int)m.size() && m[c->box] >= 0) rows.push_back(m[c->box]);
    }
    // this rank's rows, then every rank's, in rank order
    int mine = (int)rows.size();
    std::vector<int> counts(sprocs, 0), displs(sprocs, 0);
    MPI_Allgather(&mine, 1, MPI_INT, counts.data(), 1, MPI_INT, share_comm);
    int total = 0;
    for (int r = 0; r < sprocs; ++r) {
      displs[r] = total;
      total += counts[r];
    }
    std::vector<uint8_t> flags(mine);
    for (int k = 0; k < mine; ++k)
      flags[k] = IbgpuAdapter::BoxFlags(a_mesh, rows_.level[rows[k]], rows_.box[rows[k]]);
    std::vector<int> all_rows(total);
    std::vector<uint8_t> all_flags(total);
    MPI_Allgatherv(rows.data(), mine, MPI_INT, all_rows.data(), counts.data(), displs.data(),
                   MPI_INT, share_comm);
    MPI_Allgatherv(flags.data(), mine, MPI_BYTE, all_flags.data(), counts.data(), displs.data(),
                   MPI_BYTE, share_comm);
    int rc = IBGPU_OK;
    if (ibgpu_device_rank()) {
      std::vector<int64_t> r64(all_rows.begin(), all_rows.end());
      // the immersed-boundary cells' rows before the move and now
      const int last = nlev - 1;
      std::vector<int> now_ib;
      DataArray<IBCell> &mdis = a_mesh.ibarray();
      for (int i = 0; i < mdis.size(); ++i) {
        const int b = mdis[i].ci;
        if (b >= 0 && b < (int)row_of_[last].size() && row_of_[last][b] >= 0)
          now_ib.push_back(row_of_[last][b]);
      }
      for (const std::vector<int> *v : {&ib_rows_, &now_ib})
        for (int r : *v) {
          r64.push_back(r);
          all_flags.push_back(IbgpuAdapter::BoxFlags(a_mesh, rows_.level[r], rows_.box[r]));
        }
      ib_rows_.swap(now_ib);
      for (size_t k = 0; k < r64.size(); ++k) rows_.flags[r64[k]] = all_flags[k];
      rc = ibgpu_update_flags_rows(ctx_, (int64_t)r64.size(), r64.data(), all_flags.data());
      if (rc == IBGPU_OK) {
        IbgpuAdapter::FlattenImmersed(a_mesh, bodies, lists_);
        rc = IbgpuAdapter::UploadIB(ctx_, lists_);
      }
    }
    return ibgpu_share_status(rc);
  }

  // One step: ghost fills, CFL dt every dt_var_step steps, the stages and
  // the residual, aborting with the reference's code as it would.  Every
  // rank calls it and leaves with the device rank's dt.
  void TimeMarching(AMR &) {
    double r[4] = {0.0, 0.0, 0.0, 0.0};  // status, abort code, dt, CFL dt
    if (ibgpu_device_rank()) {
      ibgpu_diag diag;
      std::memset(&diag, 0, sizeof diag);
      const int rc = ibgpu_step(ctx_, ts, &dt, &diag);
      if (rc != IBGPU_OK && rc != IBGPU_E_ABORT)
        std::fprintf(stderr, "ibgpu_step: %s (%s)\n", ibgpu_errstr(rc), ibgpu_last_error());
      r[0] = rc;
      r[1] = diag.abort_code;
      r[2] = dt;
      r[3] = diag.cfl_dt;
    }
    MPI_Bcast(r, 4, MPI_DOUBLE, 0, share_comm);
    const int rc = (int)r[0];
    if (rc == IBGPU_E_ABORT) MPI_Abort(MPI_COMM_WORLD, (int)r[1]);
    if (rc != IBGPU_OK) MPI_Abort(MPI_COMM_WORLD, 1);
    dt = r[2];
    if (ts % dt_var_step == 0) CFL_dt = r[3];
  }

  // m_data <- the device state, for output, host-side forces or a regrid
  // (every rank; the device rank writes the shared arrays), and every box's
  // wall pair from the device wall distances.
  int Download() {
    if (!created_) return IBGPU_E_STATE;
    if (wall_resident_) {  // every box's pair from the device's last wall distances
      int rc = IBGPU_OK;
      if (ibgpu_device_rank()) {
        std::vector<ibgpu_wall_pairs> pr(wall_.size());
        for (size_t l = 0; l < wall_.size(); ++l) {
          IbgpuWallLevel &L = wall_[l];
          pr[l] = ibgpu_wall_pairs{L.body, L.patch, L.dist, L.sd, L.dtb, L.solid, nullptr,
                                   nullptr};
        }
        rc = ibgpu_wall_fetch(ctx_, (int)pr.size(), pr.data());
      }
      if ((rc = ibgpu_share_status(rc))) return rc;
      IbgpuAdapter::WallUnpack(a_mesh, wall_, false, nullptr, nullptr);
    }
    // the state into the shared rows (pinned), then every rank writes its
    // share of them into the mesh
    int rc = IBGPU_OK;
    if (ibgpu_device_rank()) rc = ibgpu_download_state(ctx_, rows_.prim);
    if ((rc = ibgpu_share_status(rc))) return rc;
    const int64_t nrows = rows_.n;
    for (int64_t i = nrows * srank / sprocs; i < nrows * (srank + 1) / sprocs; ++i) {
      FlowVariables &fv = a_mesh.LevelDataArray(rows_.level[i])[rows_.box[i]];
      const double *q = rows_.prim + 7 * i;
      fv.roe = q[0];
      fv.u = q[1];
      fv.v = q[2];
      fv.w = q[3];
      fv.p = q[4];
      fv.T = q[5];
      fv.e = q[6];
    }
    MPI_Barrier(share_comm);
    return IBGPU_OK;
  }

  // A level's refine/coarsen decision for AMR::TagtheBox (after Inittag):
  // the plain criterion, or with device MLP parameters the learned
  // indicator reading the device state, which is current after a step.
  // One rank: the decisions go into the level's tag lists of this process.
  int TagLevel(const ibgpu_tag_rule &rule, AMR &amr, int level, const float *d_params = nullptr) {
    if (!ctx_ || sprocs != 1) return IBGPU_E_STATE;
    return IbgpuAdapter::TagLevel(ctx_, rule, a_mesh, amr, level, d_params);
  }

  // Force and moment of every body from the device state
  // (Body::ComptWallForce): 6 per body, force then moment.
  // (every rank; the device rank's values)
  int WallForces(std::vector<double> &out) {
    if (!created_) return IBGPU_E_STATE;
    out.assign(6 * (size_t)Body::Bodynum(), 0.0);
    if (out.empty()) return IBGPU_OK;
    const int rc = ibgpu_share_status(ibgpu_device_rank() ? ibgpu_wall_forces(ctx_, out.data())
                                                          : IBGPU_OK);
    if (rc == IBGPU_OK) MPI_Bcast(out.data(), (int)out.size(), MPI_DOUBLE, 0, share_comm);
    return rc;
  }


 private:
  ibgpu_ctx *ctx_ = nullptr;  // the device rank's context
  bool created_ = false;      // on every rank once Create succeeded
  IbgpuLists lists_;          // the device rank's pair, ghost and immersed-boundary lists
  IbgpuSharedBytes rows_mem_;  // the cell rows, shared by the node's ranks
  IbgpuRows rows_;            // ... laid out in rows_mem_
  // wall_resident_: the device holds every level's wall pairs from a move
  // since the last geometry upload (the exchange buffers hold them too)
  bool device_distance_ = true, wall_check_ = false, wall_resident_ = false;
  std::vector<IbgpuWallLevel> wall_;  // exchange buffers of the device wall distances
  std::vector<std::vector<int> > row_of_;  // per level: box -> row of lists_ (-1: none)
  std::vector<int> ib_rows_;  // rows of the immersed-boundary cells after the last move
};
