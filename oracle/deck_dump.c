/*
 * deck_dump.c -- test infrastructure: parse an input deck with
 * input_deck_create and print every field of the reference's InputDeck
 * (input_deck.h:37-124), one per line.  Built twice by oracle/Makefile: once
 * against the reference's input_deck.c, once against this library's, so a
 * test can compare the two parsers on the same decks.
 */
#include <stdio.h>
#include "input_deck.h"

int main(int argc, char **argv)
{
    InputDeck *d = input_deck_create(argc > 1 ? argv[1] : NULL);
    if (!d) return 1;
    fprintf(stderr, "---\n");
#define I(f) printf(#f " %d\n", (int)d->f)
#define D(f) printf(#f " %.17g\n", d->f)
#define S(f) printf(#f " [%s]\n", d->f)
    I(nx); I(ny); I(nz); D(xmin); D(xmax); D(ymin); D(ymax); D(zmin); D(zmax);
    D(t_end); D(output_dt); D(cfl); D(gamma); D(G_const); I(problem);
    I(bc_xmin); I(bc_xmax); I(bc_ymin); I(bc_ymax); I(bc_zmin); I(bc_zmax);
    D(G_M_PNS); D(L_nu); D(g_strength); D(L_heat); S(output_dir);
    I(restart); S(restart_file); I(restart_step); D(restart_time);
    S(star1_profile); S(star2_profile);
    D(star1_x); D(star1_y); D(star1_z); D(star2_x); D(star2_y); D(star2_z);
    D(star1_vx); D(star1_vy); D(star1_vz); D(star2_vx); D(star2_vy); D(star2_vz);
    D(binary_separation); D(binary_orbital_velocity); I(binary_auto_orbit);
    S(stellar_profile); D(explosion_energy); D(explosion_radius); S(explosion_type);
    I(enable_perturbations); I(perturbation_seed);
    D(perturb_velocity_amplitude); D(perturb_velocity_kmin); D(perturb_velocity_kmax);
    I(perturb_velocity_modes); D(perturb_density_amplitude); D(perturb_density_kmin);
    D(perturb_density_kmax); I(perturb_density_modes); I(enable_sph_harmonic_mode);
    I(sph_harmonic_l); I(sph_harmonic_m); D(sph_harmonic_amp_rho); D(sph_harmonic_amp_vel);
    I(enable_torus); D(torus_major_radius); D(torus_minor_radius); D(torus_density);
    D(torus_pressure); D(torus_rotation_velocity);
    input_deck_destroy(d);
    return 0;
}
