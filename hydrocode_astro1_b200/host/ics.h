/* ics.h -- host initial conditions of the drop-in solver (internal). */
#ifndef HC_ICS_H
#define HC_ICS_H
#include "hydro_solver_3d.h"

void hc_ic_problem(GodunovHLLC3D *s, ProblemType problem);
void hc_ic_from_deck(GodunovHLLC3D *s, const InputDeck *d);
void hc_ic_log_normal(GodunovHLLC3D *s, double sigma, int seed);
State3D hc_ic_prim_to_cons(Primitive3D P, double gamma);
Primitive3D hc_ic_cons_to_prim(State3D U, double gamma);
void hc_ic_seed(int seed);
double hc_ic_uniform(void);
double hc_ic_normal(void);
/* Build a profile-based state on the device (hc_ic_profile_stars) when the
 * solver asks for it (device_ics); 0 if done, -1 to fall back to the host. */
int hc_ic_stars_device(GodunovHLLC3D *s, int nstars, const int *n, const double *const *r,
                       const double *const *rho, const double *const *u, const double *R_star,
                       const double *centre, const double *vel);
#endif
