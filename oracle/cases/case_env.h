// Environment-driven case parameters for the reference-solver oracle build
// (test infrastructure).  The reference expects every case parameter as a
// C++ global defined in a per-case "user function" file (its shipped example
// is Userfunction_cy_naca15.cpp).  The oracle case files define those globals
// and read the sizes that tests vary (grid size, levels, step count) from the
// environment, so that one oracle binary serves every test size.
//
// Globals that other translation units read during their own static
// initialisation (u_ref, T_ref, mu_ref, roe_ref, L_ref, read by
// FlowConstants.cpp) are defined with constant expressions only, so they are
// constant-initialised and the cross-TU initialisation order cannot matter.
#ifndef IB_ORACLE_CASE_ENV_H
#define IB_ORACLE_CASE_ENV_H

#include <cstdlib>
#include <cstring>

inline int case_env_int(const char *name, int dflt) {
  const char *s = std::getenv(name);
  return (s && *s) ? std::atoi(s) : dflt;
}

inline double case_env_double(const char *name, double dflt) {
  const char *s = std::getenv(name);
  return (s && *s) ? std::atof(s) : dflt;
}

#endif
