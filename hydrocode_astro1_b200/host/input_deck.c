/*
 * input_deck.c -- the `key = value` input deck of the reference
 * (input_deck.c:1-419), with the same defaults, syntax and messages, and the
 * keys this library adds.  Parsing is table driven: each key names a field
 * of InputDeck and how to convert its value.
 *
 * Syntax kept from the reference: a line is trimmed; empty lines and lines
 * starting with '#' are skipped; the key is everything before the first '='
 * (at least one character), the value everything after it (at least one
 * character, at most 255) with any '#' comment cut off; both are trimmed.
 * Integers use atoi, reals atof, booleans accept "true" or "1", strings are
 * copied truncated to their field.  Unknown keys print a warning.
 */
#include <ctype.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "input_deck.h"

static char *trim(char *s)
{
    while (isspace((unsigned char)*s)) s++;
    if (*s == 0) return s;
    char *e = s + strlen(s) - 1;
    while (e > s && isspace((unsigned char)*e)) e--;
    e[1] = '\0';
    return s;
}

static const struct { const char *name; ProblemType v; } PROBLEMS[] = {
    { "KELVIN_HELMHOLTZ", KELVIN_HELMHOLTZ }, { "BLAST_WAVE", BLAST_WAVE },
    { "RAYLEIGH_TAYLOR", RAYLEIGH_TAYLOR }, { "RIEMANN_2D", RIEMANN_2D },
    { "STALLED_SHOCK", STALLED_SHOCK }, { "STELLAR_CONVECTION", STELLAR_CONVECTION },
    { "STELLAR_PROFILE", STELLAR_PROFILE }, { "GALAXY_DISK", GALAXY_DISK },
    { "UNIFORM_DISK_TEST", UNIFORM_DISK_TEST }, { "WD_MERGER", WD_MERGER },
    { "SUPERNOVA", SUPERNOVA }, { "KELVIN_HELMHOLTZ_3D", KELVIN_HELMHOLTZ_3D },
    { "BLAST_WAVE_3D", BLAST_WAVE_3D }, { "TURBULENCE_3D", TURBULENCE_3D },
    { "SEDOV_BLAST_3D", SEDOV_BLAST_3D }, { "STELLAR_PROFILE_3D", STELLAR_PROFILE_3D },
    { "BINARY_STAR_3D", BINARY_STAR_3D },
    { "STELLAR_OCTANT_EXPLOSION_3D", STELLAR_OCTANT_EXPLOSION_3D },
    { "SOD_3D", SOD_3D }, { "POLYTROPE_3D", POLYTROPE_3D },
    { "COLD_COLLAPSE_3D", COLD_COLLAPSE_3D },
};

ProblemType parse_problem_type(const char *str)   /* input_deck.c:20-42 */
{
    for (size_t t = 0; t < sizeof PROBLEMS / sizeof PROBLEMS[0]; t++)
        if (strcmp(str, PROBLEMS[t].name) == 0) return PROBLEMS[t].v;
    fprintf(stderr, "Warning: Unknown problem type '%s', defaulting to KELVIN_HELMHOLTZ\n", str);
    return KELVIN_HELMHOLTZ;
}

BCType parse_bc_type(const char *str)   /* input_deck.c:45-52 */
{
    if (strcmp(str, "PERIODIC") == 0) return BC_PERIODIC;
    if (strcmp(str, "REFLECTIVE") == 0) return BC_REFLECTIVE;
    if (strcmp(str, "OUTFLOW") == 0) return BC_OUTFLOW;
    fprintf(stderr, "Warning: Unknown BC type '%s', defaulting to OUTFLOW\n", str);
    return BC_OUTFLOW;
}

enum Kind { K_INT, K_DBL, K_BOOL, K_STR, K_PROBLEM, K_BC, K_PRECISION, K_MOMENTS, K_WARM, K_RECON };

typedef struct {
    const char *key;
    enum Kind kind;
    size_t off;
    size_t size;   /* strings: destination size; copy at most size-1 */
} Field;

#define F(key, kind, member) { key, kind, offsetof(InputDeck, member), sizeof(((InputDeck *)0)->member) }

static const Field FIELDS[] = {
    F("nx", K_INT, nx), F("ny", K_INT, ny), F("nz", K_INT, nz),
    F("xmin", K_DBL, xmin), F("xmax", K_DBL, xmax), F("ymin", K_DBL, ymin),
    F("ymax", K_DBL, ymax), F("zmin", K_DBL, zmin), F("zmax", K_DBL, zmax),
    F("t_end", K_DBL, t_end), F("output_dt", K_DBL, output_dt), F("cfl", K_DBL, cfl),
    F("gamma", K_DBL, gamma), F("G_const", K_DBL, G_const),
    F("problem", K_PROBLEM, problem),
    F("bc_xmin", K_BC, bc_xmin), F("bc_xmax", K_BC, bc_xmax), F("bc_ymin", K_BC, bc_ymin),
    F("bc_ymax", K_BC, bc_ymax), F("bc_zmin", K_BC, bc_zmin), F("bc_zmax", K_BC, bc_zmax),
    F("G_M_PNS", K_DBL, G_M_PNS), F("L_nu", K_DBL, L_nu), F("g_strength", K_DBL, g_strength),
    F("L_heat", K_DBL, L_heat),
    F("output_dir", K_STR, output_dir),
    F("restart", K_BOOL, restart), F("restart_file", K_STR, restart_file),
    F("restart_step", K_INT, restart_step), F("restart_time", K_DBL, restart_time),
    F("star1_profile", K_STR, star1_profile), F("star2_profile", K_STR, star2_profile),
    F("star1_x", K_DBL, star1_x), F("star1_y", K_DBL, star1_y), F("star1_z", K_DBL, star1_z),
    F("star2_x", K_DBL, star2_x), F("star2_y", K_DBL, star2_y), F("star2_z", K_DBL, star2_z),
    F("star1_vx", K_DBL, star1_vx), F("star1_vy", K_DBL, star1_vy), F("star1_vz", K_DBL, star1_vz),
    F("star2_vx", K_DBL, star2_vx), F("star2_vy", K_DBL, star2_vy), F("star2_vz", K_DBL, star2_vz),
    F("binary_separation", K_DBL, binary_separation),
    F("binary_orbital_velocity", K_DBL, binary_orbital_velocity),
    F("binary_auto_orbit", K_BOOL, binary_auto_orbit),
    F("stellar_profile", K_STR, stellar_profile),
    F("explosion_energy", K_DBL, explosion_energy), F("explosion_radius", K_DBL, explosion_radius),
    F("explosion_type", K_STR, explosion_type),
    F("enable_perturbations", K_BOOL, enable_perturbations),
    F("perturbation_seed", K_INT, perturbation_seed),
    F("perturb_velocity_amplitude", K_DBL, perturb_velocity_amplitude),
    F("perturb_velocity_kmin", K_DBL, perturb_velocity_kmin),
    F("perturb_velocity_kmax", K_DBL, perturb_velocity_kmax),
    F("perturb_velocity_modes", K_INT, perturb_velocity_modes),
    F("perturb_density_amplitude", K_DBL, perturb_density_amplitude),
    F("perturb_density_kmin", K_DBL, perturb_density_kmin),
    F("perturb_density_kmax", K_DBL, perturb_density_kmax),
    F("perturb_density_modes", K_INT, perturb_density_modes),
    F("enable_sph_harmonic_mode", K_BOOL, enable_sph_harmonic_mode),
    F("sph_harmonic_l", K_INT, sph_harmonic_l), F("sph_harmonic_m", K_INT, sph_harmonic_m),
    F("sph_harmonic_amp_rho", K_DBL, sph_harmonic_amp_rho),
    F("sph_harmonic_amp_vel", K_DBL, sph_harmonic_amp_vel),
    F("enable_torus", K_BOOL, enable_torus),
    F("torus_major_radius", K_DBL, torus_major_radius),
    F("torus_minor_radius", K_DBL, torus_minor_radius),
    F("torus_density", K_DBL, torus_density), F("torus_pressure", K_DBL, torus_pressure),
    F("torus_rotation_velocity", K_DBL, torus_rotation_velocity),
    /* added keys */
    F("grav_omega", K_DBL, grav_omega), F("grav_tolerance", K_DBL, grav_tolerance),
    F("grav_max_iter", K_INT, grav_max_iter), F("grav_lmax", K_INT, grav_lmax),
    F("precision", K_PRECISION, precision), F("grav_moments", K_MOMENTS, moment_order),
    F("warm_start", K_WARM, warm_start), F("unet_weights", K_STR, unet_weights),
    F("max_steps", K_INT, max_steps), F("log_every", K_INT, log_every),
    F("log_normal_noise", K_DBL, log_noise), F("sor_depth", K_INT, sor_depth),
    F("checkpoint_every", K_INT, checkpoint_every), F("checkpoint_file", K_STR, checkpoint_file),
    F("reconstruction", K_RECON, recon), F("device_ics", K_INT, device_ics),
    F("unet_guard", K_INT, unet_guard),
};

static void set_defaults(InputDeck *d)   /* input_deck.c:63-153 */
{
    memset(d, 0, sizeof *d);
    d->nx = d->ny = d->nz = 128;
    d->xmin = d->ymin = d->zmin = -1.0;
    d->xmax = d->ymax = d->zmax = 1.0;
    d->t_end = 1.0;
    d->output_dt = 0.1;
    d->cfl = 0.4;
    d->gamma = 5.0 / 3.0;
    d->G_const = 1.0;
    d->problem = KELVIN_HELMHOLTZ_3D;
    d->bc_xmin = d->bc_xmax = d->bc_ymin = d->bc_ymax = d->bc_zmin = d->bc_zmax = BC_PERIODIC;
    strcpy(d->output_dir, "output");
    strcpy(d->star1_profile, "stellar_profile_1.txt");
    strcpy(d->star2_profile, "stellar_profile_2.txt");
    d->star1_x = -1.5; d->star2_x = 1.5;
    d->star1_vy = 0.5; d->star2_vy = -0.5;
    d->binary_separation = 3.0;
    d->binary_auto_orbit = true;
    strcpy(d->stellar_profile, "stellar_profile.txt");
    d->explosion_energy = 1.0;
    d->explosion_radius = 0.2;
    strcpy(d->explosion_type, "thermal");
    d->perturbation_seed = 42;
    d->perturb_velocity_amplitude = 0.01;
    d->perturb_velocity_kmin = 1.0;
    d->perturb_velocity_kmax = 10.0;
    d->perturb_velocity_modes = 20;
    d->perturb_density_amplitude = 0.01;
    d->perturb_density_kmin = 1.0;
    d->perturb_density_kmax = 10.0;
    d->perturb_density_modes = 20;
    d->sph_harmonic_l = 1;
    d->sph_harmonic_m = 0;
    d->sph_harmonic_amp_rho = 0.05;
    d->sph_harmonic_amp_vel = 0.05;
    d->torus_major_radius = 1.2;
    d->torus_minor_radius = 0.2;
    d->torus_density = 1.0;
    d->torus_pressure = 0.1;
    /* added keys */
    d->grav_omega = 1.5;
    d->grav_tolerance = 1.0e-6;
    d->grav_max_iter = 10000;
    d->log_every = 10;
    strcpy(d->checkpoint_file, "checkpoint.ckpt");
    d->device_ics = -1;
    d->unet_guard = 3;
}

static int is_true(const char *v) { return strcmp(v, "true") == 0 || strcmp(v, "1") == 0; }

static void assign(InputDeck *d, const Field *f, const char *v)
{
    char *p = (char *)d + f->off;
    switch (f->kind) {
    case K_INT: *(int *)p = atoi(v); break;
    case K_DBL: *(double *)p = atof(v); break;
    case K_BOOL: *(bool *)p = is_true(v) ? true : false; break;
    case K_STR: strncpy(p, v, f->size - 1); p[f->size - 1] = '\0'; break;
    case K_PROBLEM: *(ProblemType *)p = parse_problem_type(v); break;
    case K_BC: *(BCType *)p = parse_bc_type(v); break;
    case K_PRECISION:
        *(int *)p = (strcmp(v, "fp32") == 0 || strcmp(v, "mixed") == 0 || strcmp(v, "1") == 0) ? 1 : 0;
        break;
    case K_MOMENTS: *(int *)p = (strcmp(v, "tree") == 0 || strcmp(v, "1") == 0) ? 1 : 0; break;
    case K_WARM: *(int *)p = (strcmp(v, "unet") == 0 || strcmp(v, "1") == 0) ? 1 : 0; break;
    case K_RECON: *(int *)p = (strcmp(v, "plm") == 0 || strcmp(v, "muscl") == 0 || strcmp(v, "1") == 0) ? 1 : 0; break;
    }
}

InputDeck *input_deck_create(const char *filename)   /* input_deck.c:55-326 */
{
    InputDeck *d = (InputDeck *)malloc(sizeof(InputDeck));
    if (!d) {
        fprintf(stderr, "Error: Failed to allocate memory for InputDeck\n");
        return NULL;
    }
    set_defaults(d);
    if (filename == NULL) {
        printf("No input file provided, using defaults.\n");
        return d;
    }
    FILE *fp = fopen(filename, "r");
    if (!fp) {
        fprintf(stderr, "Warning: Could not open input file '%s', using defaults.\n", filename);
        return d;
    }
    printf("Reading input deck from: %s\n", filename);
    char line[512];
    int line_num = 0;
    while (fgets(line, sizeof line, fp)) {
        line_num++;
        char *t = trim(line);
        if (*t == '\0' || *t == '#') continue;
        char *eq = strchr(t, '=');
        if (!eq || eq == t) continue;             /* no key */
        if (eq[1] == '\0' || eq[1] == '\n') continue;   /* no value */
        char key[128], val[256];
        size_t kl = (size_t)(eq - t);
        if (kl > 127) continue;                    /* key longer than the reference accepts */
        memcpy(key, t, kl);
        key[kl] = '\0';
        /* value: up to 255 characters, stops at a newline */
        size_t vl = strcspn(eq + 1, "\n");
        if (vl > 255) vl = 255;
        memcpy(val, eq + 1, vl);
        val[vl] = '\0';
        char *hash = strchr(val, '#');
        if (hash) *hash = '\0';
        char *k = trim(key), *v = trim(val);
        const Field *hit = NULL;
        for (size_t q = 0; q < sizeof FIELDS / sizeof FIELDS[0]; q++)
            if (strcmp(k, FIELDS[q].key) == 0) { hit = &FIELDS[q]; break; }
        if (hit) assign(d, hit, v);
        else fprintf(stderr, "Warning: Unknown parameter '%s' on line %d\n", k, line_num);
    }
    fclose(fp);
    printf("Successfully loaded input deck.\n");
    return d;
}

void input_deck_destroy(InputDeck *deck) { free(deck); }

static const char *bcname(BCType b)
{
    return b == BC_PERIODIC ? "PERIODIC" : (b == BC_REFLECTIVE ? "REFLECTIVE" : "OUTFLOW");
}

void input_deck_print(const InputDeck *d)   /* input_deck.c:336-420 */
{
    printf("\n==============================================\n");
    printf("INPUT DECK PARAMETERS\n");
    printf("==============================================\n");
    printf("Grid:\n");
    printf("  nx = %d, ny = %d, nz = %d\n", d->nx, d->ny, d->nz);
    printf("  x: [%.2f, %.2f]\n", d->xmin, d->xmax);
    printf("  y: [%.2f, %.2f]\n", d->ymin, d->ymax);
    printf("  z: [%.2f, %.2f]\n", d->zmin, d->zmax);
    printf("\nTime:\n");
    printf("  t_end = %.3f\n", d->t_end);
    printf("  output_dt = %.3f\n", d->output_dt);
    printf("  cfl = %.3f\n", d->cfl);
    printf("\nPhysics:\n");
    printf("  gamma = %.3f\n", d->gamma);
    printf("  G_const = %.3f\n", d->G_const);
    printf("\nProblem: ");
    const char *pn = "OTHER";
    for (size_t t = 0; t < sizeof PROBLEMS / sizeof PROBLEMS[0]; t++)
        if (PROBLEMS[t].v == d->problem) pn = PROBLEMS[t].name;
    printf("%s\n", pn);
    printf("\nBoundary Conditions:\n");
    printf("  x: %s / %s\n", bcname(d->bc_xmin), bcname(d->bc_xmax));
    printf("  y: %s / %s\n", bcname(d->bc_ymin), bcname(d->bc_ymax));
    printf("  z: %s / %s\n", bcname(d->bc_zmin), bcname(d->bc_zmax));
    printf("\nOutput:\n");
    printf("  Directory: %s\n", d->output_dir);
    if (d->restart) {
        printf("\nRestart:\n");
        printf("  File: %s\n", d->restart_file);
        printf("  Step: %d\n", d->restart_step);
        printf("  Time: %.3f\n", d->restart_time);
    }
    printf("\nGravity solver: omega = %.3f, tolerance = %.3e, max_iter = %d, lmax = %d\n",
           d->grav_omega, d->grav_tolerance, d->grav_max_iter, d->grav_lmax);
    printf("Device path: %s hydro, %s moments, warm start %s\n", d->precision ? "fp32" : "fp64",
           d->moment_order ? "tree" : "sequential", d->warm_start ? "unet" : "previous potential");
    printf("==============================================\n\n");
}
