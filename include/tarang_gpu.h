/*
 * tarang_gpu.h — C ABI of the B200 pseudo-spectral time-step path of Tarang-4.0.
 *
 * The reference has no FFI layer: its "operator API" is the C++ class interface that the
 * solver drivers call (trunk/src/IFluid/Ifluid_main.cc:258-301, IMHD/IMHD_main.cc,
 * RBslip/RB_slip_main.cc:365-400).  Each entry point below replaces one of those calls; the
 * header-only C++ mirror classes in tarang_b200.hpp (CVF, CSF, IncVF, IncSF, IncFluid) keep
 * the reference's method and member names and call these functions.
 *
 * Conventions
 *  - Every function returns an int status: TG_OK (0) or a negative TG_ERR_* code.  The last
 *    error text of a context is available from tg_last_error().
 *  - Host buffers are caller-owned.  Device state is owned by the context.
 *  - Fields cross the boundary in the reference layout: complex<double> interleaved (re, im),
 *    row-major [l1][l2][l3] with l3 in [0, N3/2]; real space uses the same buffer as
 *    N1 x N2 x (N3+2) doubles with the last two reals of each row as zeroed padding
 *    (lib/four/four_tr.cc:299-302).  n_doubles = 2 * N1 * N2 * (N3/2+1).
 *  - A context is externally synchronised (like the reference's single-threaded rank):
 *    different contexts may be used from different threads.  All work of a context is
 *    queued on its stream; calls that return data to the host synchronise that stream.
 */
#ifndef TARANG_GPU_H
#define TARANG_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TG_ABI_VERSION 1

/* status codes */
#define TG_OK 0
#define TG_ERR_ARG (-1)         /* invalid argument or unsupported size */
#define TG_ERR_OOM (-2)         /* device allocation failed / request over the HBM budget */
#define TG_ERR_NONFINITE (-3)   /* total energy is NaN or Inf (Ifluid_main.cc:282-286) */
#define TG_ERR_CUDA (-4)        /* a CUDA runtime call failed */
#define TG_ERR_UNSUPPORTED (-5) /* combination not implemented */
#define TG_ERR_TIMEOUT (-6)     /* a bounded wait ran out */
#define TG_ERR_STATE (-7)       /* call out of order (e.g. Time_advance before Compute_nlin) */
#define TG_ERR_BUSY (-8)        /* serving: no slot or no memory free right now */

/* basis_type (string_switches[1] in the reference) */
#define TG_FOUR 0
#define TG_SCFT 1
/* program kind (prog_para.d: INC_FLUID, INC_MHD, INC_SCALAR, RB_SLIP) */
#define TG_FLUID 0
#define TG_MHD 1
#define TG_SCALAR 2
#define TG_RB 3
/* arithmetic form */
#define TG_FP64 0
#define TG_FP32_MIXED 1 /* FP32 transforms and products, FP64 RK state/projection/reductions */
/* integ_scheme (IncFluid::Time_advance time_advance.cc:60-163): integrating-factor Euler, the
 * integrating-factor midpoint rule and the integrating-factor RK4 (Lawson) */
#define TG_EULER 1
#define TG_RK2 2
#define TG_RK4 4
/* force_field_proc (compute_force_main.cc:43-124) */
#define TG_FORCE_DECAY 0
#define TG_FORCE_ENERGY_SUPPLY 1  /* Compute_force_const_energy_helicity_supply (FOUR; fluid, MHD,
                                     passive scalar): force_para = inner, outer, eps, eps_h/(k eps),
                                     then eps_B, epsh_B/(k eps_B) (MHD) or eps_T (scalar) */
#define TG_FORCE_ENERGY_HELICITY 2  /* Compute_force_const_energy_helicity (compute_force_const_ek_hk.cc,
                                       FOUR; fluid, MHD, passive scalar): force_para = inner, outer,
                                       energy level, H/(k E), then the B level and H/(k E) of B (MHD)
                                       or the scalar level (scalar) */
#define TG_FORCE_MODES 5      /* a fixed force on given modes, set by tg_set_force_modes: the
                                 Taylor-Green, ABC and given-mode forcings (force_field_proc 3, 4, 5) */
#define TG_FORCE_CORIOLIS 21  /* Force = V x Omega, Omega = force_para[0..2], evaluated from each RK
                                 stage's velocity (compute_force_Coriolis.cc:47-80) */
#define TG_FORCE_LIQUID_METAL 101 /* Compute_force_Liquid_metal (compute_force_LM.cc:46-70), FOUR fluid:
                                     Force = -(B0 . K)^2 / K^2 V, B0 = force_para[0..2], from each RK
                                     stage's velocity */
#define TG_FORCE_RB 51
#define TG_FORCE_RB_ROTATION 52  /* convection with rotation (compute_force_RB.cc:132-195): the
                                    buoyancy of TG_FORCE_RB plus c V x Omega, Omega =
                                    force_para[0..2], c = Pr (PRLARGE, USMALL), 1 (PRSMALL, USMALL)
                                    or sqrt(Pr/Ra) (ULARGE) */

#define TG_RB_PRLARGE 0
#define TG_RB_PRSMALL 1
#define TG_RB_ULARGE 0
#define TG_RB_USMALL 1

/* field ids (dense, reference layout) */
#define TG_V1 0 /* U.V1..V3 */
#define TG_V2 1
#define TG_V3 2
#define TG_W1 3 /* W.V1..V3 (B field of MHD) */
#define TG_W2 4
#define TG_W3 5
#define TG_T 6 /* T.F (scalar / temperature) */
#define TG_NLIN1 7 /* U.nlin1..3 */
#define TG_NLIN2 8
#define TG_NLIN3 9
#define TG_WNLIN1 10
#define TG_WNLIN2 11
#define TG_WNLIN3 12
#define TG_TNLIN 13
#define TG_PRESSURE 14 /* NLIN's CSF F: the pressure */
#define TG_FORCE1 15   /* U.Force1..3 */
#define TG_FORCE2 16
#define TG_FORCE3 17
#define TG_WORK0 24 /* TG_WORK0 .. TG_WORK0+7: free dense work fields for the transforms */
#define TG_NWORK 8
#define TG_NFIELDS 32

/* energy-transfer kinds (compute_flux.cc, compute_shell_tr.cc) */
#define TG_ET_UU 0 /* U< -> U> (fluid, and U->U of MHD) */
#define TG_ET_BB 1 /* B< -> B> */
#define TG_ET_UB 2 /* U< -> B> */
#define TG_ET_BU 3 /* B< -> U> */
#define TG_ET_TT 4 /* T< -> T> (passive scalar, FOUR) */
#define TG_ET_ZP 5 /* Z+< -> Z+> with Z- as helper (MHD Elsasser, flux_Elsasser) */
#define TG_ET_ZM 6 /* Z-< -> Z-> with Z+ as helper (MHD Elsasser, W.flux_Elsasser) */

typedef struct tg_config {
  int N[3];           /* N1, N2, N3 (N3 even) */
  int basis;          /* TG_FOUR / TG_SCFT */
  int physics;        /* TG_FLUID / TG_MHD / TG_SCALAR / TG_RB */
  int precision;      /* TG_FP64 / TG_FP32_MIXED */
  int dealias;        /* 1: alias_switch "DEALIAS" (2/3 rule), 0: "ALIAS" */
  int scheme;         /* TG_EULER / TG_RK2 / TG_RK4 */
  double kfactor[3];  /* 2 pi / L per axis (Ifluid_main.cc:159-161) */
  double nu;          /* dissipation_coefficient of U */
  double eta;         /* dissipation_coefficient of B (MHD) */
  double kappa;       /* diffusion_coefficient of T */
  double dt;          /* Tdt: the upper bound of Get_dt (compute_dt.cc:47-59) */
  int force_kind;     /* TG_FORCE_* */
  double force_para[6]; /* force_double_para(1..6) of the force_field_proc (see TG_FORCE_*) */
  int n_shells;       /* energy transfer: no_shells (= no_spheres), scheme 0 radii */
  double rb_ra, rb_pr;  /* Rayleigh and Prandtl numbers (RB) */
  int device;         /* CUDA device ordinal */
  void* stream;       /* cudaStream_t to queue on; NULL: the context creates one */
  /* RB nondimensionalisation (RB_slip_main.cc:222-262, compute_force_RB.cc:50-105):
   * Pr_switch TG_RB_PRLARGE / TG_RB_PRSMALL, RB_Uscaling TG_RB_ULARGE / TG_RB_USMALL, and
   * temperature_grad (+1 convection, -1 stable stratification; solver_double_para(6)) */
  int rb_pr_switch;
  int rb_u_scaling;
  double rb_temp_grad;
  /* hyper_dissipation_coefficient of U and B, hyper_diffusion_coefficient of T: the viscous
   * factor exp(-nu K^2 dt) becomes exp(-(nu + nu_h K^2) K^2 dt) (Mult_field_exp_ksqr_dt
   * mult_exp_visc.cc:56-165, Array_exp_ksqr_FOUR four_basic.cc:377-403); 0: off (the
   * hyper_dissipation_switch / hyper_diffusion_switch of the reference) */
  double hyper_nu, hyper_eta, hyper_kappa;
} tg_config;

typedef struct tg_ctx tg_ctx;

/* defaults: FOUR fluid FP64 DEALIAS RK4, kfactor 1, decay forcing, 12 shells, device 0 */
void tg_config_default(tg_config* cfg);

int tg_ctx_create(const tg_config* cfg, tg_ctx** out);
int tg_ctx_destroy(tg_ctx* ctx);
const char* tg_last_error(const tg_ctx* ctx);
int tg_synchronize(tg_ctx* ctx);
/* bytes of device memory the context holds */
int tg_device_bytes(const tg_ctx* ctx, size_t* bytes);

/* Field I/O in the reference layout (Read_data_MPI / Write_data_MPI array_basic.cc:294-858
 * without the MPI gather).  With dealias on, uploads of solver fields keep the 2/3 support
 * only (the reference dealiases every initial condition, init_cond_*.cc): for the state fields
 * (V, W, T) only those modes cross the bus, as up to four strided copies into the solver's
 * compact rows.  tg_field_download writes every entry (zeros outside the support). */
int tg_field_upload(tg_ctx* ctx, int field, const double* host, size_t n_doubles);
int tg_field_download(tg_ctx* ctx, int field, double* host, size_t n_doubles);
/* A state field's stored (dealiased) modes only, into the caller's dense reference-layout
 * array; its other entries are left as they are.  For a driver that keeps the fields in host
 * memory between steps, where those entries are zero already (as in the reference after
 * Dealias): the transfer is the stored 30 % of the array (no counterpart in the reference). */
int tg_field_download_stored(tg_ctx* ctx, int field, double* host, size_t n_doubles);
int tg_field_copy(tg_ctx* ctx, int dst_field, int src_field);
/* A work field of its own for the caller (the reference's temporary arrays, e.g. the
 * VF_temp / VF_temp_r fields IncVF.h:75-531 allocates): reserves a free slot among
 * TG_WORK0 .. TG_WORK0+7, allocates its dense device array (zeroed), returns its id in *field;
 * TG_ERR_BUSY when all eight are reserved.  tg_field_free releases the slot and its memory. */
int tg_field_alloc(tg_ctx* ctx, int* field);
int tg_field_free(tg_ctx* ctx, int field);

/* Field files in the reference's text format (host memory, no context; the solver mirror moves
 * fields between them and a context).  tg_write_field_file: IncFluid::Output_field
 * (lib/IncFluid/output/output_field.cc:43-108) with Write_data_MPI / Write_data_kz0plane_MPI
 * (lib/fields/array_fn/array_basic.cc:814-898): "%% Time = t", then each field as "(re,im) " per
 * mode in [l1][l2][l3] order at 12 significant digits, two newlines after each.  fields are the
 * state fields in reference order (V1 V2 V3, then W1 W2 W3 or T), each 2*N1*N2*(N3/2+1) doubles;
 * vx_vy = 1 (output_vx_vy_switch) writes the kz = 0 plane only of V3 (and W3).  append = 1 adds
 * to an existing file.
 * tg_read_field_file: IncFluid::Init_cond (lib/IncFluid/input/init_cond_field.cc:47-88, 179-223)
 * with Read_data_MPI (array_basic.cc:294-383); lines starting with '%' are skipped; with vx_vy = 1
 * V3 (and W3) for kz >= 1 come from incompressibility (IncVF::Last_component
 * lib/IncFlow/misc/field_k_fns.cc:79-87).  TG_ERR_ARG on a short or malformed file. */
int tg_write_field_file(const char* path, double time, const int N[3], int n_fields,
                        const double* const* fields, int vx_vy, int append);
int tg_read_field_file(const char* path, const int N[3], int basis, const double kfactor[3], int n_fields,
                       double* const* fields, int vx_vy);
/* Reduced-size field files: the low-wavenumber corner Nr[3] (Nr <= N; FOUR: Nr1 even; Nr2, Nr3
 * even) of N-grid fields, as IncFluid::Output_field_reduced writes it with Write_data_MPI /
 * Write_data_kz0plane_MPI (output_field.cc:505-600, array_basic.cc:997-1347: rows kx = 0..Nr1/2
 * then -Nr1/2+1..-1 (SCFT 0..Nr1-1), ky likewise, kz 0..Nr3/2, values "(re,im)" with no
 * separator) and Init_cond_reduced reads it (init_cond_field.cc:294-338, array_basic.cc:388-715:
 * the +Nr/2 rows also fill -Nr/2; everything outside the corner is zero; vx_vy as above). */
int tg_write_field_file_reduced(const char* path, double time, const int N[3], const int Nr[3], int basis,
                                int n_fields, const double* const* fields, int vx_vy, int append);
int tg_read_field_file_reduced(const char* path, const int N[3], const int Nr[3], int basis, const double kfactor[3],
                               int n_fields, double* const* fields, int vx_vy);

/* Forward_transform_array / Inverse_transform_array (universal_tr.cc:66-146) on a work field,
 * in place.  parity: 0 cos/even, 1 sin/odd (SCFT only; ignored for FOUR). */
int tg_forward_transform(tg_ctx* ctx, int field, int parity);
int tg_inverse_transform(tg_ctx* ctx, int field, int parity);

/* IncFluid::Compute_force() (compute_force_main.cc:43-124) */
int tg_compute_force(tg_ctx* ctx);
/* IncVF::Compute_nlin() / (W) / (T)  (compute_nlin.cc:58-108, compute_nlin_VF_MHD.cc:72-164,
 * compute_nlin_SF.cc:65-263); nlin is dealiased */
int tg_compute_nlin(tg_ctx* ctx);
/* IncFluid::Add_force() (add_force.cc:47-84): nlin -= Force */
int tg_add_force(tg_ctx* ctx);
/* The fixed force of TG_FORCE_MODES (Setup_Taylor_Green_force_field, Setup_ABC_force_field,
 * Compute_force_given_modes_SIMPLE: lib/IncFlow/misc/force_model.cc:57-170,
 * lib/IncFluid/force/compute_force_modes.cc:97-250): n modes, k[3 i + 0..2] = (kx, ky, kz)
 * wavenumber indices (FOUR: kx, ky signed; SCFT: kx >= 0; kz >= 0; each at most
 * TG_FORCE_MODES_KMAX in magnitude) of modes the context stores, F[2 nstate i + 2 c + 0..1] =
 * (Re, Im) of the force on state field c there (V1, V2, V3, then W1..W3 of MHD or T of a
 * scalar).  Every other mode has no force; a mode listed twice takes its last value.  Replaces
 * the previous set (n = 0 clears it).  TG_ERR_STATE unless force_kind is TG_FORCE_MODES. */
#define TG_FORCE_MODES_KMAX 64
int tg_set_force_modes(tg_ctx* ctx, int n, const int* k, const double* F);
/* IncVF::Compute_pressure() (compute_pressure.cc:54-62) */
int tg_compute_pressure(tg_ctx* ctx);
/* IncFluid::Compute_rhs() (compute_rhs.cc:52-149) */
int tg_compute_rhs(tg_ctx* ctx);
/* IncFluid::Get_dt() (compute_dt.cc:47-108); also sets the dt Time_advance uses */
int tg_get_dt(tg_ctx* ctx, double* dt);
/* IncFluid::Time_advance() RK4 (time_advance.cc:100-155): precondition as in the reference,
 * nlin = N(u) - f and pressure computed for the current field. */
int tg_time_advance(tg_ctx* ctx);
/* n iterations of the loop body Ifluid_main.cc:261-286 (force, nlin, add force, pressure,
 * Get_dt, Time_advance, energy).  energies (may be NULL) receives the total energy after each
 * step (n doubles; for MHD the sum U + B).  Returns TG_ERR_NONFINITE if an energy is NaN/Inf. */
int tg_step(tg_ctx* ctx, int n, double* energies);
/* elapsed simulated time and step count since creation */
int tg_time(const tg_ctx* ctx, double* t, long long* steps);

/* CV_Compute_totalenergy_diss (Cvf.cc:385-397) of group 0 = U, 1 = B, 2 = T (T: CSF energy) */
int tg_energy(tg_ctx* ctx, int group, double* energy, double* dissipation);
/* CV_Compute_shell_spectrum (Cvf.cc:419-449): ek = [3][n] per component (group T: [1][n]),
 * dissk = [n] (may be NULL).  n must be >= kmax_outside + 1. */
int tg_shell_spectrum(tg_ctx* ctx, int group, double* ek, double* dissk, int n);
/* Anisotropic spectra of the velocity (group 0) or magnetic field (group 1, MHD), FOUR or SCFT,
 * about the anisotropy axis `axis` (1 x, 2 y, 3 z: globalvar_anisotropy_switch).
 * tg_ring_spectrum: CVF::CV_Compute_ring_spectrum (fields/Cvf.cc:484-504 with
 * Compute_local_ring_spectrum_FOUR four/four_energy.cc:828-955): spherical shells 0 .. kmax
 * (Max_radius_inside) x polar sectors 0 .. n_sectors of equal angle up to pi/2 (Cvf.cc:84-100,
 * Get_sector_index basis_basicfn.cc:304-320); ek1 sums mult |(V x K)_axis / K_perp|^2 (on the
 * axis, the first transverse component), ek2 the rest of mult |V|^2, dissk = 2 (S1 + S2) with a
 * K^2 weight.  tg_cylinder_ring_spectrum: CV_Compute_cylinder_ring_spectrum (Cvf.cc:537-559
 * with four_energy.cc:1450-1516): cylindrical shells ceil(K_perp) 0 .. Anis_max_Krho_radius_inside
 * x slabs 0 .. n_slabs of equal |K_par| up to Anis_max_Kpll (Cvf.cc:168-190, Get_slab_index
 * basis_basicfn.cc:373-390); ek1 sums mult |V_axis|^2, ek2 the rest.  Arrays are
 * [shells][n + 1] row-major (column 0 stays empty as in the reference); n = capacity of each
 * array in doubles; ek2, dissk may be NULL.  n_sectors, n_slabs <= TG_RING_MAX_SECTORS.
 * For axis 3 the reference's on-axis and cylinder branches test the axis-2 switch twice (an
 * uninitialised value); the z-axis components are used.
 * SCFT (Compute_local_ring_spectrum_SCFT / _cylinder_ scft/scft_energy.cc:814-940, 1423-1480):
 * kx >= 0, Multiplicity_factor_SCFT, V = (-i V1, V2, V3), on-axis components (V2, V3),
 * (V3, -i V1), (-i V1, V2) for axes 1, 2, 3, the SCFT box (kx up to 2 N1/3 dealiased, N1 - 1
 * aliased; Anis_max_Kpll_SCFT's dealiased y extent is (N2/2) kf as written there).  As written
 * in the reference, the off-axis modes of the SCFT spherical ring spectrum (ek1, ek2, dissk)
 * carry no multiplicity factor. */
#define TG_RING_MAX_SECTORS 64
int tg_ring_sizes(tg_ctx* ctx, int axis, int* ring_shells, int* cylinder_shells);
/* Helicity spectra: modal helicity 2 mult K . (Vr x Vi) per mode (shell form FOUR; ring forms
 * FOUR and SCFT, scft_energy.cc:1334-1370, 1794-1830, with V = (-i V1, V2, V3)).
 * tg_shell_spectrum_helicity: CVF::CV_Compute_shell_spectrum_helicity (Cvf.cc:640-646,
 * Compute_shell_spectrum_helicity_FOUR four/four_energy.cc:551-651): the three terms
 * 2 mult K_i (Vr x Vi)_i in h1, h2, h3 over shells 0 .. Min_radius_outside (n >= that + 1),
 * shells beyond Max_radius_inside rescaled by Approx_number_modes_in_shell / (sum of 2 mult
 * over the shell).  tg_ring_spectrum_helicity / tg_cylinder_ring_spectrum_helicity:
 * CV_Compute_ring_spectrum_helicity / CV_Compute_cylinder_ring_spectrum_helicity (Cvf.cc:648-665,
 * four_energy.cc:1357-1450, 1825-1910), binned as tg_ring_spectrum / tg_cylinder_ring_spectrum. */
int tg_shell_spectrum_helicity(tg_ctx* ctx, int group, double* h1, double* h2, double* h3, int n);
int tg_ring_spectrum_helicity(tg_ctx* ctx, int group, int axis, int n_sectors, double* h, int n);
int tg_cylinder_ring_spectrum_helicity(tg_ctx* ctx, int group, int axis, int n_slabs, double* h, int n);
int tg_ring_spectrum(tg_ctx* ctx, int group, int axis, int n_sectors, double* ek1, double* ek2, double* dissk, int n);
int tg_cylinder_ring_spectrum(tg_ctx* ctx, int group, int axis, int n_slabs, double* ek1, double* ek2, double* dissk,
                              int n);
/* Ring-to-ring energy transfer (IncVF::Compute_ring_tr, EnergyTrdir/compute_ring_tr.cc:60-90 and
 * the MHD kinds :174-215; Fill_array_ring universal_ET.cc:70-100, Local_ring_mult_all_FOUR
 * four/four_ET.cc:330-386; SCFT Local_ring_mult_all_SCFT scft/scft_ET.cc:273-346 with the SCFT
 * products and derivatives of the shell transfers): tr[i][j][m][s], (n_ring_shells+1) x (n_sectors+1) x
 * (n_ring_shells+1) x (n_sectors+1) doubles, is the transfer from giver ring (shell i =
 * 1..n_ring_shells-1, sector j = 1..n_sectors) to receiver ring (m, s).  kind TG_ET_UU
 * (ring_to_ring_self), for MHD TG_ET_BB (W.ring_to_ring_self), TG_ET_UB (ring_to_ring_VF, U to
 * B), TG_ET_ZP and TG_ET_ZM (ring_to_ring_Elsasser, W.ring_to_ring_Elsasser;
 * compute_ring_tr.cc:226-285), and for a passive scalar TG_ET_TT (ring_to_ring_SF,
 * Compute_ring_tr_scalar :104-131).  TG_ET_BU has no ring table in the reference (TG_ERR_ARG).  Ring radii: scheme 0 (EnergyTr.cc:190-210; tg_ring_radii), 5 <=
 * n_ring_shells <= 32; sectors of equal angle up to pi/2 about `axis`.  As in the reference, a
 * giver ring holds only the modes with theta <= pi/2 (K_par >= 0), while receivers fold theta. */
int tg_ring_radii(tg_ctx* ctx, int n_ring_shells, double* radii, int n);
int tg_ring_to_ring(tg_ctx* ctx, int kind, int axis, int n_ring_shells, int n_sectors, double* tr, int n);
/* Cylinder-ring-to-ring transfer (IncVF::Compute_cylinder_ring_tr, EnergyTrdir/
 * compute_cylin_ring_tr.cc:53-80; Fill_array_cylinder_ring universal_ET.cc:100-125,
 * Local_cyl_ring_mult_all_FOUR four/four_ET.cc:422-530, _SCFT scft_ET.cc:436-478): as tg_ring_to_ring with cylindrical
 * shells of K_perp (scheme 0 radii up to Anis_max_Krho_radius_inside, EnergyTr.cc:300-320;
 * tg_cylinder_radii) and slabs of K_par of equal width up to Anis_max_Kpll in place of sectors.
 * A giver holds the modes with K_par >= 0 (the reference compares the signed K_par); receivers
 * take |K_par|.  The reference sets the middle radii only when no_ring_shells > 5; here
 * whenever n_cylinder_shells > 5. */
int tg_cylinder_radii(tg_ctx* ctx, int axis, int n_cylinder_shells, double* radii, int n);
int tg_cylinder_ring_to_ring(tg_ctx* ctx, int kind, int axis, int n_cylinder_shells, int n_slabs, double* tr, int n);
/* shell radii of the energy transfer (EnergyTr.cc:136-160): n_shells + 1 doubles */
int tg_et_radii(tg_ctx* ctx, double* radii, int n);
/* Compute_flux (compute_flux.cc:52-304): flux[s], s = 0..n_shells (index 0 unused); kind
 * TG_ET_UU/BB/UB/BU, TG_ET_ZP/ZM (Elsasser, :228-255) or TG_ET_TT (Compute_flux_scalar :82-95;
 * convection: Compute_flux_RB).  FOUR and SCFT (Shell_mult_single_SCFT / Shell_mult_all_SCFT
 * scft/scft_ET.cc:53-265: Kmagnitude_SCFT, Multiplicity_factor_SCFT, x derivatives of the sine and
 * cosine product series). */
int tg_flux(tg_ctx* ctx, int kind, double* flux, int n);
/* Compute_shell_tr (compute_shell_tr.cc:59-281): n is the table's dimension (>= n_shells + 1);
 * tr holds n x n doubles, row-major, giver shell by row, receiver shell by column */
int tg_shell_to_shell(tg_ctx* ctx, int kind, double* tr, int n);
/* IncVF::Compute_kinetic_helicity_flux (EnergyTrdir/compute_helicity_flux.cc:47-75), FOUR: the
 * helicity flux out of each sphere s = 1 .. n_shells of the energy-transfer radii,
 * -P(U.grad U<, omega>)/2 - P(U.grad omega<, U>)/2 + P(omega.grad U<, U>)/2 with omega = i K x U,
 * X< the field inside the sphere and P(N, R>) = sum over |K| > R_s of 2 mult Re(N . R*)
 * (Prod_out_sphere_nlinV / Prod_out_sphere_nlin_vorticity prod_nlinV.cc:62-150).  n >= n_shells + 1. */
int tg_helicity_flux(tg_ctx* ctx, double* flux, int n);
/* IncVF::Compute_magnetic_helicity_flux (EnergyTrdir/compute_helicity_flux.cc:94-135), FOUR MHD:
 * the magnetic helicity flux out of each sphere s = 1 .. n_shells, P(B.grad U<, a>)/2
 * - P(U.grad B<, a>)/2 + P(U x B<, B>)/2 with a = i K x B / K^2
 * (Prod_out_sphere_nlin_vector_potential prod_nlinV.cc:154-162, Shell_mult_vector_potential_FOUR
 * four_ET.cc:905-965; U x B< of EnergyTr_Compute_nlin_UcrossB ET_compute_nlin.cc:317-337).
 * n >= n_shells + 1. */
int tg_magnetic_helicity_flux(tg_ctx* ctx, double* flux, int n);
/* IncVF::Compute_kinetic_helicity_shell_tr (compute_helicity_shell_tr.cc:56-109) and
 * Compute_magnetic_helicity_shell_tr (:114-172), FOUR: the three terms of the fluxes above with the
 * giver held to shell n = 1 .. n_shells-1 (R_{n-1} < |K| <= R_n) and the receivers binned by shell
 * over |K| <= R_in (Shell_mult_all_FOUR, Shell_mult_vorticity_all_FOUR,
 * Shell_mult_vector_potential_all_FOUR four_ET.cc:181-256, 999-1090, 1094-1190).  tr is n x n
 * row-major, n >= n_shells + 1.  The reference's K = 0 entry of the vector-potential sum is 0/0;
 * here a(0) = 0. */
int tg_helicity_shell_to_shell(tg_ctx* ctx, double* tr, int n);
int tg_magnetic_helicity_shell_to_shell(tg_ctx* ctx, double* tr, int n);
/* Get_Nusselt_no (nusselt.cc:53-89), RB only */
int tg_nusselt(tg_ctx* ctx, double* nusselt);
/* IncVF::Compute_force_feed_shell (lib/IncFlow/EnergyTrdir/compute_force_feed.cc:70-76, with
 * Shell_mult_all_FOUR lib/four/four_ET.cc:181-226): energy fed by the force into each shell,
 * feed[i] = sum over |K| <= R_in with Get_shell_index(|K|) = i of 2 mult Re(F . V*), i = 0..S
 * (n >= S+1), with the force last computed (tg_compute_force, or the last RK stage of tg_step;
 * computed from the current field if the context never computed one) and the current field.
 * Zero for a decaying run.  FOUR; fluid, MHD and passive scalar (the velocity's feed). */
int tg_force_feed(tg_ctx* ctx, double* feed, int n);
/* The force feed of one field group: 0 the velocity (as tg_force_feed), 1 the magnetic field of
 * an MHD context (W.forceV_shell of Compute_force_feed_shell(W)), 2 the passive scalar
 * (forceSF_shell of Compute_force_feed_shell_scalar, Re(F_T . T*)) (compute_force_feed.cc:70-155).
 * FOUR; fluid, MHD and passive scalar.  With the liquid-metal force the velocity feed is
 * sum 2 mult Re(F . V*) = -2 mult (B0 . K)^2/K^2 |V|^2 per shell.  Convection (FOUR or SCFT;
 * Compute_force_feed_shell_RB, PRLARGE / PRSMALL): group 0 the buoyancy fu theta against u1,
 * group 2 ft u1 against theta. */
int tg_force_feed_group(tg_ctx* ctx, int group, double* feed, int n);
/* IncVF::Compute_force_feed_ring / Compute_force_feed_cylinder_ring (compute_force_feed.cc:162-300,
 * Ring_mult_all / Cyl_ring_mult_all four_ET.cc:335-386, 492-530): the force feed 2 mult Re(F . X*)
 * of field group 0 (velocity), 1 (B, MHD) or 2 (passive scalar) binned by receiver ring
 * (cylinder = 0: tg_ring_radii shells x n_sectors polar sectors) or cylinder ring (cylinder = 1:
 * tg_cylinder_radii shells x n_sectors K_par slabs) about `axis`; out is
 * [n_ring_shells + 1][n_sectors + 1] row-major (n >= that many).  FOUR, or an SCFT band forcing
 * (Ring_mult_all_SCFT scft_ET.cc:273-346); no convection. */
int tg_force_feed_ring(tg_ctx* ctx, int group, int cylinder, int axis, int n_ring_shells, int n_sectors, double* out,
                       int n);

/* ------------------------------------------------------------------------------------------
 * Allocation-free energy reduction.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory: an in-situ diagnostic called from inside
 * another code's time loop, where the host application owns all device memory through its own
 * pool and does not allow cudaMalloc (it synchronises the device and can fail part-way through
 * a long run).  Such a caller holds its spectral fields in its own device buffers and needs
 * the energy and dissipation of those fields without a tg_ctx.
 *
 * Computes, for each of n_fields consecutive fields at d_fields (device memory, reference
 * layout, 2*N1*N2*(N3/2+1) doubles each), the FOUR total energy (Get_total_energy_FOUR) and
 * dissipation 2*sum mult K^2 |A|^2 (Get_total_Sn_FOUR with n = 2, Cvf.cc:385-397), and writes
 * d_out[2f] = energy of field f, d_out[2f+1] = dissipation of field f (device memory,
 * 2*n_fields doubles).  The same numbers tg_energy returns for a context's fields.
 *
 * No cudaMalloc/cudaFree or allocating library call: the per-block partial sums live in a
 * fixed device array of 8 x 1184 x 2 doubles (151,552 bytes) that every GPU loading this library
 * holds until exit.  Limit: 1 <= n_fields <= TG_NOALLOC_MAX_FIELDS; anything beyond returns
 * TG_ERR_ARG.  d_fields must lie on a 16-byte boundary (the fields are read as 16-byte complex
 * values) and d_out on an 8-byte boundary; otherwise TG_ERR_ARG.  The first call in a CUDA
 * context looks up that array's device address in the context current on the calling thread
 * and caches it per context (keyed on the context's unique id, so a reset device or a caller's
 * own context gets its own lookup): make that first call before any stream capture.
 * Work is queued on `stream` (cudaStream_t; NULL = default stream) and the call returns
 * without waiting.  Every call shares the array and it keeps the last call's partials; calls
 * that overlap on the GPU (different streams, or concurrent host threads) race on it.
 * ---------------------------------------------------------------------------------------- */
#define TG_NOALLOC_MAX_FIELDS 8
int tg_energy_noalloc(const double* d_fields, int n_fields, const int N[3], const double kfactor[3],
                      int dealias, double* d_out, void* stream);

/* ------------------------------------------------------------------------------------------
 * Profiling (no counterpart in the reference, whose only timing is time(0) around main,
 * src/main.cc:95-151): per-launch CUDA events on the context's stream.  While enabled, steps
 * run eagerly (no graph replay).  Stats aggregate by kernel name; algorithmic bytes are the
 * bytes a launch must read and write on the stored (2/3-dealiased) support.
 * ---------------------------------------------------------------------------------------- */
typedef struct tg_kernel_stat {
  char name[48];
  int launches;
  double total_ms;
  double bytes_per_launch;
} tg_kernel_stat;

int tg_profile_enable(tg_ctx* ctx, int enable);
/* synchronises; fills up to max stats, sets *n; clears the records */
int tg_profile_read(tg_ctx* ctx, tg_kernel_stat* out, int max, int* n);

/* ------------------------------------------------------------------------------------------
 * Failure-path test hook (no counterpart in the reference, which has no bounded waits).
 *
 * The TMA-staged transform passes wait for each tile with a bounded number of polls; a block
 * whose wait runs out skips its tile (its output is not written), waits again with the full
 * limit so that its copy lands before it leaves, and sets the context's status word.  The next
 * call that synchronises the context (tg_step after each chunk, tg_synchronize, downloads,
 * energies, spectra, transfer tables, ...) then returns TG_ERR_TIMEOUT with a message in
 * tg_last_error and clears the word: the fields written since the last check are not valid,
 * the context itself stays usable.  In the serving loop the requests of that batch fail with
 * TG_ERR_TIMEOUT.
 *
 * TG_DEBUG_SHORT_TMA_WAIT (value 1 / 0) gives the first wait for a tile no polls at all, so
 * every TMA-staged block reports a timeout; value 0 restores the normal limit.  Changing it
 * drops the context's captured step graph.  For tests of the failure path only.
 * ---------------------------------------------------------------------------------------- */
#define TG_DEBUG_SHORT_TMA_WAIT 1
int tg_debug_set(tg_ctx* ctx, int what, long long value);

/* ------------------------------------------------------------------------------------------
 * Serving (no counterpart in the reference, whose programs run one solve per process,
 * src/main.cc:95-151): a request loop that admits independent solves by an HBM budget, keeps
 * their spectral state resident and advances requests of the same shape together.
 *
 * Requests whose configurations agree on everything but the coefficients (nu, eta, kappa, Ra,
 * Pr, dt) share a batch: one context with B slots whose kernels take the slot as a grid
 * dimension, so one launch of each pass (and one CUDA graph per step) advances all of them.
 * Each slot's arithmetic is the same as that of a lone context: a request's fields after n
 * steps do not depend on what else is resident (bit for bit), and equal tg_step's.  Forced
 * requests (TG_FORCE_ENERGY_SUPPLY) get a context of their own.
 *
 * One host thread drives a server; calls on one server must not overlap.
 * ---------------------------------------------------------------------------------------- */
typedef struct tg_server tg_server;

/* ------------------------------------------------------------------ slab-sharded solve
 * One solve split over `world` ranks (one process per GPU), the reference's MPI slab
 * decomposition (basis_basicfn.cc:49-281): rank r's context holds compact kx rows
 * [xs[r], xs[r] + xn[r]) of the stored modes (a near-equal split of the nkx stored rows), and
 * between the two exchanges of an RHS evaluation the real y planes [ys[r], ys[r] + yn[r]).  The
 * caller moves the data between the phases (an NCCL all-to-all, or device copies when several
 * ranks share a GPU) and sums the reductions; per RK stage s = 1..4 of a step:
 *   tg_slab_phase(ctx, 0, s)   y-inverse of the stage input, packed: TG_SLAB_INV_SEND field f
 *                              holds world chunks [xn[r]][yn[d]][kzp], chunk d for rank d
 *   all-to-all of each input field f: chunk r of every rank's INV_SEND, in rank order, into
 *                              TG_SLAB_INV_RECV f = [nkx][yn[r]][kzp]
 *   tg_slab_phase(ctx, 1, s)   x-inverse, fused z-pass, x-forward: TG_SLAB_FWD_SEND product q =
 *                              [nkx][yn[r]][kzp], chunk d = the rows of rank d, [xn[d]][yn[r]][kzp]
 *   all-to-all of each product q into TG_SLAB_FWD_RECV q = world chunks [xn[r]][yn[s]][kzp]
 *   tg_slab_phase(ctx, 2, s)   unpack, y-forward, the RK stage on the rank's modes; after
 *                              stage 4 the rank's 8 reduction sums are in TG_SLAB_SUMS
 * then the element-wise sum of every rank's TG_SLAB_SUMS into TG_SLAB_GLOBAL_SUMS and
 * tg_slab_phase(ctx, 3, 0): Get_dt (compute_dt.cc:47-55) and the time and step count.  Before
 * the first step (after tg_slab_upload): phase 4 (the state's sums into TG_SLAB_SUMS), the same
 * sum, and phase 5 (dt only).  Elements are complex values of elem_bytes (16 FP64, 8 FP32-mixed);
 * every buffer is device memory on the context's stream.  Built for fluid, passive scalar and
 * convection with forces local in K (none, buoyancy, Coriolis, liquid metal, fixed modes): the
 * band forcings and MHD return TG_ERR_UNSUPPORTED.  A slab context answers only tg_slab_* calls,
 * tg_ctx_destroy and tg_last_error. */
#define TG_SLAB_MAX_RANKS 64
#define TG_SLAB_INV_SEND 0
#define TG_SLAB_INV_RECV 1
#define TG_SLAB_FWD_SEND 2
#define TG_SLAB_FWD_RECV 3
#define TG_SLAB_SUMS 4        /* double[8] */
#define TG_SLAB_GLOBAL_SUMS 5 /* double[8] */
typedef struct tg_slab_info {
  int world, rank;
  int x0, nx, y0, ny;              /* this rank's kx rows and y planes */
  int xs[TG_SLAB_MAX_RANKS], xn[TG_SLAB_MAX_RANKS];
  int ys[TG_SLAB_MAX_RANKS], yn[TG_SLAB_MAX_RANKS];
  int nkx, nky, nkz, kzp;          /* stored modes: the compact layout [nkx][nky][kzp] */
  int nin, nprod;                  /* fields of the inverse and forward exchanges */
  size_t elem_bytes;
} tg_slab_info;
int tg_slab_create(const tg_config* cfg, int world, int rank, tg_ctx** out);
int tg_slab_info_get(const tg_ctx* ctx, tg_slab_info* info);
int tg_slab_buffer(tg_ctx* ctx, int which, int field, void** ptr);
int tg_slab_phase(tg_ctx* ctx, int phase, int stage);
/* state field f (V1..V3, then T) in the reference layout [N1][N2][N3/2+1] complex: upload
 * keeps the rank's stored rows, download writes them (other rows of host untouched) */
int tg_slab_upload(tg_ctx* ctx, int field, const double* host);
int tg_slab_download(tg_ctx* ctx, int field, double* host);
/* the reductions after phase 3 or 5 (sums[0] energy of U, sums[1] sum mult K^2 |U|^2, [4], [5]
 * the same of T) and scalars [0] dt, [1] time, [2] steps, [3] non-finite flag */
int tg_slab_scalars(tg_ctx* ctx, double* sums, double* scalars);

typedef struct tg_server_config {
  size_t hbm_budget_bytes; /* admission budget: device bytes of all resident batches */
  int max_batch;           /* most requests in one batch */
  int device;
  int use_graphs;          /* 1: replay one captured CUDA graph per batch and active count */
  int keep_results;        /* 1: keep each finished request's fields for tg_server_result, in
                              device memory outside the batch budget (page-locked host memory
                              where the device has no room) until tg_server_release */
  /* 1: tg_server_submit keeps the caller's init pointer instead of copying the fields; the
   * caller keeps that memory valid and unchanged until the request leaves TG_REQ_QUEUED (its
   * admission copies straight from it to the device).  0: submit copies (into page-locked
   * memory when the pool has room). */
  int borrow_inputs;
} tg_server_config;

typedef struct tg_request {
  tg_config cfg;        /* shape, physics, precision, coefficients (device and stream ignored) */
  int n_steps;          /* RK4 steps to run */
  const double* init;   /* initial fields, reference layout, concatenated per state field
                           (fluid 3, MHD 6, scalar/RB 4); copied at submit */
  size_t n_doubles;     /* length of init */
} tg_request;

#define TG_REQ_QUEUED 0
#define TG_REQ_RUNNING 1
#define TG_REQ_DONE 2
#define TG_REQ_FAILED 3

typedef struct tg_request_status {
  int state;            /* TG_REQ_* */
  int error;            /* TG_ERR_* when failed: TG_ERR_OOM (does not fit the budget),
                           TG_ERR_NONFINITE (energy not finite), TG_ERR_CUDA */
  int steps_done;
  double submit_s, start_s, finish_s; /* server clock (seconds) */
  double final_energy;  /* kinetic energy after the last step (MHD: kinetic + magnetic) */
  double t_final;       /* simulated time */
} tg_request_status;

typedef struct tg_server_stats {
  size_t bytes_resident;   /* device bytes of the resident batches */
  size_t bytes_peak;
  int n_batches;           /* resident batches */
  int n_running, n_queued;
  long long rounds;        /* pump rounds that advanced at least one batch */
  long long request_steps; /* steps advanced, summed over requests */
  long long graph_launches, eager_steps;
} tg_server_stats;

/* device bytes that a batch of `batch` requests of configuration cfg holds (admission cost) */
int tg_request_bytes(const tg_config* cfg, int batch, size_t* bytes);

int tg_server_create(const tg_server_config* cfg, tg_server** out);
int tg_server_destroy(tg_server* srv);
/* validates and copies the request; TG_ERR_ARG / TG_ERR_UNSUPPORTED for a configuration that
 * tg_ctx_create rejects or an init of the wrong length (no id).  A request that cannot fit the
 * budget even alone gets an id and state TG_REQ_FAILED with TG_ERR_OOM. */
int tg_server_submit(tg_server* srv, const tg_request* req, long long* id);
/* one scheduling round: advance the resident batches (one after another on the device, each on
 * its own stream) by one step, or with graphs on by as many steps as fit in the slowest running
 * batch's step (at most 16, never past a request's last step); meanwhile admit queued requests
 * that fit
 * (first come first served, later ones may pass one that waits for room); then retire finished
 * and failed requests.  *n_active = requests running or queued afterwards */
int tg_server_pump(tg_server* srv, int* n_active);
/* tg_server_pump in two halves, so that the caller's own host work overlaps the round's steps on
 * the device: pump_begin launches the round (TG_ERR_STATE when a round is already open);
 * submissions, polls and results may follow; pump_end admits queued requests (those submitted
 * in between included), waits for the round and retires finished requests, as tg_server_pump.
 * pump_end without an open round is an admission-only round.  tg_server_drain and
 * tg_server_destroy close an open round first. */
int tg_server_pump_begin(tg_server* srv);
int tg_server_pump_end(tg_server* srv, int* n_active);
/* pump until every submitted request is done or failed (bounded by max_rounds; 0 = no bound) */
int tg_server_drain(tg_server* srv, long long max_rounds);
int tg_server_poll(tg_server* srv, long long id, tg_request_status* st);
/* final fields of a finished request (keep_results = 1), same packing as tg_request.init: copied
 * from the device when called (the batches' streams go on meanwhile) */
int tg_server_result(tg_server* srv, long long id, double* host, size_t n_doubles);
/* drop a finished request's kept fields (their device memory is freed once any copy of them
 * has run; no host wait) */
int tg_server_release(tg_server* srv, long long id);
/* ids of requests that finished (done or failed) since the last call, oldest first: up to max
 * of them into ids, *n = how many were written */
int tg_server_take_finished(tg_server* srv, long long* ids, int max, int* n);
int tg_server_stats_get(tg_server* srv, tg_server_stats* st);
/* One entry per resident batch: its shape and physics, slot capacity, active requests and the
 * device time of one batch step (CUDA events on the batch's stream around the steps of its last
 * timed round, averaged over rounds at the same active count) with the active count it was
 * taken at.  Up to max entries into out; *n = entries written. */
typedef struct tg_batch_stat {
  int N[3];
  int basis, physics, precision;
  int capacity;          /* request slots of the batch */
  int n_active;          /* requests running in it now */
  int step_ms_n_active;  /* active requests during the timed steps (0: none timed yet) */
  double step_ms;        /* device ms of one step of the whole batch */
  double device_ms;      /* device ms of all the batch's steps so far (CUDA events) */
  long long steps;       /* batch steps run so far */
} tg_batch_stat;
int tg_server_batch_stats(tg_server* srv, tg_batch_stat* out, int max, int* n);
double tg_server_clock(tg_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* TARANG_GPU_H */
