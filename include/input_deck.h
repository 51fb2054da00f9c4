/*
 * input_deck.h -- the reference's `key = value` input deck (input_deck.h of
 * the reference project), kept field for field so the reference driver
 * main_3d.c compiles unchanged against it.  Keys this library adds are
 * appended after the reference's fields; the reference parser only warns on
 * them (input_deck.c:317), so extended decks stay readable by both.
 *
 * Reference interfaces: InputDeck (input_deck.h:37-124), ProblemType
 * (:8-27), BCType (:30-34), input_deck_create/destroy/print,
 * parse_problem_type, parse_bc_type (:127-131).
 */
#ifndef INPUT_DECK_H
#define INPUT_DECK_H

#include <stdbool.h>
#include <stdio.h>

/* Problem types: the reference's values in their order, then additions. */
typedef enum {
    KELVIN_HELMHOLTZ,
    BLAST_WAVE,
    RAYLEIGH_TAYLOR,
    RIEMANN_2D,
    STALLED_SHOCK,
    STELLAR_CONVECTION,
    STELLAR_PROFILE,
    GALAXY_DISK,
    UNIFORM_DISK_TEST,
    WD_MERGER,
    SUPERNOVA,
    KELVIN_HELMHOLTZ_3D,
    BLAST_WAVE_3D,
    TURBULENCE_3D,
    SEDOV_BLAST_3D,
    STELLAR_PROFILE_3D,
    BINARY_STAR_3D,
    STELLAR_OCTANT_EXPLOSION_3D,
    /* additions */
    SOD_3D,                 /* Sod tube along x: rho,p = 1,1 | 0.125,0.1 */
    POLYTROPE_3D,           /* n=1 polytrope, hydrostatic, centred */
    COLD_COLLAPSE_3D        /* rho ~ 1/r sphere, e = 0.05 GM/R */
} ProblemType;

typedef enum {
    BC_PERIODIC,
    BC_REFLECTIVE,
    BC_OUTFLOW
} BCType;

typedef struct {
    /* Grid */
    int nx, ny, nz;
    double xmin, xmax;
    double ymin, ymax;
    double zmin, zmax;

    /* Time */
    double t_end;
    double output_dt;
    double cfl;

    /* Physics */
    double gamma;
    double G_const;

    ProblemType problem;

    BCType bc_xmin, bc_xmax;
    BCType bc_ymin, bc_ymax;
    BCType bc_zmin, bc_zmax;

    double G_M_PNS;
    double L_nu;
    double g_strength;
    double L_heat;

    char output_dir[256];

    bool restart;
    char restart_file[256];
    int restart_step;
    double restart_time;

    /* BINARY_STAR_3D */
    char star1_profile[256];
    char star2_profile[256];
    double star1_x, star1_y, star1_z;
    double star2_x, star2_y, star2_z;
    double star1_vx, star1_vy, star1_vz;
    double star2_vx, star2_vy, star2_vz;
    double binary_separation;
    double binary_orbital_velocity;
    bool binary_auto_orbit;

    /* STELLAR_OCTANT_EXPLOSION_3D */
    char stellar_profile[256];
    double explosion_energy;
    double explosion_radius;
    char explosion_type[32];

    /* perturbations */
    bool enable_perturbations;
    int perturbation_seed;
    double perturb_velocity_amplitude;
    double perturb_velocity_kmin;
    double perturb_velocity_kmax;
    int perturb_velocity_modes;
    double perturb_density_amplitude;
    double perturb_density_kmin;
    double perturb_density_kmax;
    int perturb_density_modes;
    bool enable_sph_harmonic_mode;
    int sph_harmonic_l;
    int sph_harmonic_m;
    double sph_harmonic_amp_rho;
    double sph_harmonic_amp_vel;

    /* torus */
    bool enable_torus;
    double torus_major_radius;
    double torus_minor_radius;
    double torus_density;
    double torus_pressure;
    double torus_rotation_velocity;

    /* ---- keys added by this library (appended) ---- */
    double grav_omega;          /* grav_omega     (default 1.5) */
    double grav_tolerance;      /* grav_tolerance (default 1e-6) */
    int grav_max_iter;          /* grav_max_iter  (default 10000) */
    int grav_lmax;              /* grav_lmax: 0 = reference monopole + quadrupole */
    int precision;              /* precision = fp64 | fp32 (0 / 1) */
    int moment_order;           /* grav_moments = sequential | tree (0 / 1) */
    int warm_start;             /* warm_start = prev | unet (0 / 1) */
    char unet_weights[256];     /* unet_weights = path */
    int max_steps;              /* max_steps: stop after this many steps (0 = no cap) */
    int log_every;              /* log_every  (default 10, the reference's cadence) */
    double log_noise;           /* log_normal_noise: sigma of exp(sigma N(0,1)) on rho */
    int sor_depth;              /* sor_depth: SOR kernels, as hc_config.sor_depth (0 = default) */
    int checkpoint_every;       /* checkpoint_every: binary checkpoint every N steps (0 = off) */
    char checkpoint_file[256];  /* checkpoint_file (default checkpoint.ckpt; the latest one is kept) */
    int recon;                  /* reconstruction = constant | plm (MUSCL-Hancock, fp64 only) */
    int device_ics;             /* device_ics: profile set-ups on the device (1), host (0), auto (-1, default) */
    int unet_guard;             /* unet_guard: learned-start outcome monitor, consecutive losses that
                                   switch the network off (default 3; 0 = off) */
} InputDeck;

InputDeck *input_deck_create(const char *filename);
void input_deck_destroy(InputDeck *deck);
void input_deck_print(const InputDeck *deck);
ProblemType parse_problem_type(const char *str);
BCType parse_bc_type(const char *str);

#endif /* INPUT_DECK_H */
