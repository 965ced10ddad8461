// Oracle case: isentropic vortex on a single-level periodic Cartesian grid
// (the flux/stage bandwidth workload: N x N cells on [0,10]^2, inviscid,
// vortex strength 5 advected at Mach 0.5 and 45 degrees).
//
// Test infrastructure only.  This file plays the role of the reference's
// per-case user file (Userfunction_cy_naca15.cpp): it defines every global
// and hook the reference solver expects from a case, for this workload.
//
// Inviscid flow: the reference hard-enables its viscous terms
// (NS_Solver.H:15 "#define VISCOUSITY").  Setting mu_ref = 0 makes
// Re = roe_ref*u_ref*L_ref/mu_ref infinite (FlowConstants.cpp:6), so every
// viscous stress and heat flux is exactly zero (NS_Solver.cpp:568-583) and
// the update reduces bit-for-bit to the inviscid one.
//
// Environment: IB_NX (cells per side, default 64).
#include <cmath>
#include <string>
#include <vector>

#include "AMR.H"
#include "AMRSpaceTime.H"
#include "BCValues.H"
#include "Body.H"
#include "Domain.H"
#include "FlowVariables.H"
#include "InputFunc.H"
#include "Pltoutput.H"
#include "case_env.h"

using namespace std;

// ---- time-step control (AMRSpaceTime.H) ---------------------------------
double dt = 1.0;  // large: the first CFL evaluation sets dt (dt = min(CFL_dt, dt*dt_ratio))
double t_sum = 1.0e30;
const int ts_sum = 1 << 30;
const double CFL = case_env_double("IB_CFL", 0.5);
const double dt_ratio = 1.0;
int dt_var_step = 1;
const int dts_plt = 1 << 30;
const int dts_time_var = 1 << 30;
const int dts_space_var = 1 << 30;

// ---- mesh ------------------------------------------------------------------
const int max_mesh_level = 1;
const int init_level_num = 1;
const Point lowpt = Point(0, 0, 0);
const Point highpt = Point(case_env_int("IB_NX", 64), case_env_int("IB_NX", 64), 1);
static const double kDomainLength = 10.0;

string meshfile = "none";
Pointxyz meshscale(1.0, 1.0, 1.0);
Pointxyz frame_rotate_vel = Pointxyz(0.0, 0.0, 0.0);
Pointxyz frame_rotate_origin = Pointxyz(0.0, 0.0, 0.0);
Pointxyz frame_trans_vel = Pointxyz(0.0, 0.0, 0.0);
const bool moveflag = false;

// ---- reference scales (constant-initialised; see case_env.h) --------------
double roe_ref = 1.0;
double L_ref = 1.0;
double mu_ref = 0.0;  // inviscid: Re = inf
double u_ref = 1.0;
double T_ref = 1.0 / (0.5 * 0.5 * 287.4 * 1.4);  // Ma = u_ref/sqrt(gama*Rg_ref*T_ref) = 0.5

bool additional_output = false;
const int init_jump = 0;
const int filenodenum = 1;
const int filelevelnum = 1;
const int filebodynum = 0;
const char soln_file_name[30] = "none";

// ---- vortex parameters ----------------------------------------------------
static const double kVortexBeta = 5.0;
static const double kVortexXc = 5.0, kVortexYc = 5.0;
static const double kAdvectAngle = 45.0 / 180.0 * 3.14159265358979323846;

void AMR::ADPRule(vector<Body> &) {
  adpflag = false;
  for (int i = 0; i < max_mesh_level; ++i) {
    m_level[i].torefine = false;
    m_level[i].toderefine = false;
  }
}

void AMR::SetRefineFlag() {}

// single-level case: nothing to tag, nothing to dump
FILE *g_oracle_tag_dump = nullptr;
int g_oracle_tag_pass = 0;

void AMR::TagtheBox(const int &ilevel, vector<Body> &) { m_level[ilevel].Inittag(); }

void Body::Motion_Rule(Mesh &, double &) {}

void SetTwodFlag() {
  level_twod_flag.resize(max_mesh_level);
  level_twod_flag[0] = false;
  for (int i = 1; i < max_mesh_level; ++i) level_twod_flag[i] = true;
}

void InitSpaceParams() {
  double h = kDomainLength / double(highpt.xy[0]);
  double dh0[3] = {h, h, 0.1};
  periodic[0] = true;
  periodic[1] = true;
  periodic[2] = true;
  ComptLevelgridsize(dh0);
}

void Body::SetBodyParams(vector<Body> &, Mesh &, vector<Body> &) {}

void Domain::SetBlockNum() { blocknum = Point(1, 1, 1); }

void Domain::SetFaceProperty(DataArray<Box> &, DataArray<BoxCellGeom> &) {
  facenum = 6;
  faceup.resize(facenum);
  facedown.resize(facenum);
  facetype.resize(facenum);
  facedir.resize(facenum);
  refboxface.resize(facenum);
  faceup[0] = Point(0, 99999, 99999);
  facedown[0] = Point(-10, -99999, -99999);
  facedir[0] = Point(1, 0, 0);
  faceup[1] = Point(boxnum.ix() + 10, 99999, 99999);
  facedown[1] = Point(boxnum.ix() - 1, -99999, -99999);
  facedir[1] = Point(-1, 0, 0);
  faceup[2] = Point(99999, 0, 99999);
  facedown[2] = Point(-99999, -10, -99999);
  facedir[2] = Point(0, 1, 0);
  faceup[3] = Point(99999, boxnum.iy() + 10, 99999);
  facedown[3] = Point(-99999, boxnum.iy() - 1, -99999);
  facedir[3] = Point(0, -1, 0);
  faceup[4] = Point(99999, 99999, 0);
  facedown[4] = Point(-99999, -99999, -10);
  facedir[4] = Point(0, 0, 1);
  faceup[5] = Point(99999, 99999, boxnum.iz() + 10);
  facedown[5] = Point(-99999, -99999, boxnum.iz() - 1);
  facedir[5] = Point(0, 0, -1);
  for (int i = 0; i < facenum; ++i) facetype[i] = -99;
  CheckPeriodicFaceType();
}

void BCValues::SetBCType_125_Inputinletbdlayer(FlowVariables &, FlowVariables &, const int &,
                                               double &, int &, Mesh &) {}

void BCValues::SetInitValues() {
  inlet_flow_angle = kAdvectAngle;
  initvar.u = cos(kAdvectAngle);
  initvar.v = sin(kAdvectAngle);
  initvar.w = 0.0;
  double speed = pow(pow(initvar.u, 2) + pow(initvar.v, 2) + pow(initvar.w, 2), 0.5);
  initvar.T = pow(speed / Ma, 2) / (gama * Rg);
  initvar.roe = 1.0;
  Get_p_ideal_gas(initvar);
  Get_E(initvar);
}

// Isentropic vortex (Shu's form, perturbation velocity scaled by the free
// stream sound speed over sqrt(gamma), temperature by the free-stream T).
void BCValues::UserInit(Mesh &amesh, const int &ilevel, const int &bn) {
  FlowVariables fv;
  double x = amesh.bc(ilevel, bn)[0] - kVortexXc;
  double y = amesh.bc(ilevel, bn)[1] - kVortexYc;
  double r2 = x * x + y * y;
  double cinf = sqrt(gama * Rg * initvar.T);
  double uscale = cinf / sqrt(gama);
  double amp = kVortexBeta / (2.0 * 3.14159265358979323846) * exp(0.5 * (1.0 - r2));
  fv.u = initvar.u - amp * y * uscale;
  fv.v = initvar.v + amp * x * uscale;
  fv.w = 0.0;
  double dT = -(gama - 1.0) * kVortexBeta * kVortexBeta /
              (8.0 * gama * 3.14159265358979323846 * 3.14159265358979323846) * exp(1.0 - r2);
  fv.T = initvar.T * (1.0 + dT);
  fv.roe = initvar.roe * pow(fv.T / initvar.T, 1.0 / (gama - 1.0));
  Get_p_ideal_gas(fv);
  Get_E(fv);
  amesh.LevelBoxData(ilevel, bn) = fv;
}

void BCValues::SetBDFaceVars() {}

void BCValues::SetBackPressure(Mesh &) { backpressure = 0.0; }

void Pltoutput::Design_User_File() { userfilenum = 0; }

void Pltoutput::Print_Var_as_Func_of_Time(vector<Body> &, NS_Solver &) {}

void Pltoutput::Print_Var_as_Func_of_Space(vector<Body> &) {}

void Mesh::ComptSectionAvePre(const int &, double &p0, double &T0, int) {
  p0 = 0.0;
  T0 = 0.0;
}
