"""CPU oracle (test infrastructure only) of the spectral post-processing after
the forward transform: the divergence of a flux vector (the reference's
u.grad(T) term is -div(u T)), the curl of u x B (the induction term), and the
curl and divergence of the momentum forces (the vorticity equation's inertia
and Lorentz terms, the pressure source).

Restates, in plain numpy:
- const_sph_scalar_advect (MHD_src/sph_MHD/const_sph_divergence.f90:49-74);
- the interior rows, cal_sph_nod_vect_div2
  (MHD_src/sph_MHD/cal_sph_exp_rotation.f90:254-290):
      div(j,k) = (sum_s d1(k,s) S(j,k+s) - dS/dr(j,k)) * max(g3(j), 1/2) / r_k^2;
- the fixed-field boundary rows, cal_sph_div_flux_4_fix_in / _fix_out
  (MHD_src/sph_MHD/cal_sph_exp_fixed_scalar.f90:381-456), where the boundary
  node's S is replaced by the caller's fixed value;
- the radial FDM coefficients: 3x3 Taylor matrices inverted by cofactors,
  nod_r_2nd_fdm_coef_noequi (CORE_src/SPH_SPECTR_src/set_radius_func_noequi.f90:193-260),
  copy_fdm2_nod_coefs_from_mat (CORE_src/SPH_SPECTR_src/t_fdm_coefs.f90:146-163),
  cal_fdm2_coef_fix_fld_ICB / _CMB (MHD_src/sph_MHD/cal_fdm_coefs_4_boundaries.f90:155-190, 256-290),
  cal_inverse_33_matrix and cal_det_33_matrix (CORE_src/BASE/cal_inverse_small_matrix.f90:57-80, 176-215);
- 1/r^2 as (1/r)^2 (CORE_src/SPH_SPECTR_src/set_radius_4_sph_dynamo.f90:105).

- const_sph_force_rot2 (MHD_src/sph_MHD/const_sph_rotation.f90:225-250), the
  curl of a force with the velocity boundary rows of sel_bc_sph_vorticity
  (MHD_src/sph_MHD/select_exp_velocity_bc.f90:215-262): non-slip rows
  cal_sph_nod_icb_rigid_rot2 / cal_sph_nod_cmb_rigid_rot2
  (set_sph_exp_rigid_ICB.f90:159-197, set_sph_exp_rigid_CMB.f90:129-166) with
  cal_fdm2_coef_fix_df_ICB / _CMB (cal_fdm_coefs_4_boundaries.f90:195-231,
  297-334); free-slip rows cal_sph_nod_icb_free_rot2 / cal_sph_nod_cmb_free_rot2
  (set_sph_exp_free_ICB.f90:131-166, set_sph_exp_free_CMB.f90) with
  cal_fdm2_ICB_free_vp / _vt and cal_fdm2_CMB_free_vp / _vt
  (coef_fdm2_free_ICB.f90, coef_fdm2_free_CMB.f90);
- const_sph_div_force (const_sph_divergence.f90:79-108): the divergence rows
  with the boundary node's own value, cal_sph_nod_nobc_in_div2 / _out_div2
  (cal_sph_exp_nod_none_bc.f90:153-185, 309-341).

Parity unpinned against the reference's own outputs (no Fortran compiler in
this image); the tests pin this restatement by the FDM being exact for
quadratic radial profiles.
"""
import numpy as np


def _det22(a):
    return a[0, 0] * a[1, 1] - a[1, 0] * a[0, 1]


def _det33(a):
    det = 0.0
    for k in range(3):
        cols = [c for c in range(3) if c != k]
        t = a[1:3][:, cols]
        det = det + (-1) ** k * _det22(t) * a[0, k]
    return det


def inverse33(a):
    """cal_inverse_33_matrix: a_inv(kj, ki) = (-1)^(ki+kj) det(minor(ki, kj)) / det(a)."""
    a = np.asarray(a, dtype=np.float64)
    a_det = 1.0 / _det33(a)
    inv = np.zeros((3, 3))
    for kj in range(3):
        for ki in range(3):
            rows = [r for r in range(3) if r != ki]
            cols = [c for c in range(3) if c != kj]
            t = a[rows][:, cols]
            inv[kj, ki] = (-1) ** (ki + kj) * _det22(t) * a_det
    return inv


def fdm_coefs(radius):
    """(d1[k, 0..2] for the offsets -1, 0, +1 at interior k; icb[0..2] for
    nodes kr_in, kr_in+1, kr_in+2; cmb[0..2] for kr_out, kr_out-1, kr_out-2)."""
    r = np.asarray(radius, dtype=np.float64)
    nr = len(r)
    d1 = np.zeros((nr, 3))
    for k in range(1, nr - 1):
        dp, dn = r[k + 1] - r[k], r[k] - r[k - 1]
        t = np.array([[1.0, 0.0, 0.0], [1.0, dp, 0.5 * dp * dp], [1.0, -dn, 0.5 * dn * dn]])
        inv = inverse33(t)
        d1[k] = [inv[1, 2], inv[1, 0], inv[1, 1]]  # S(k-1), S(k), S(k+1)
    dp1, dp2 = r[1] - r[0], r[2] - r[0]
    t = np.array([[1.0, 0.0, 0.0], [1.0, dp1, dp1 * dp1 / 2.0], [1.0, dp2, dp2 * dp2 / 2.0]])
    icb = inverse33(t)[1, :]
    dn1, dn2 = r[-1] - r[-2], r[-1] - r[-3]
    t = np.array([[1.0, 0.0, 0.0], [1.0, -dn1, dn1 * dn1 / 2.0], [1.0, -dn2, dn2 * dn2 / 2.0]])
    cmb = inverse33(t)[1, :]
    return d1, icb, cmb


def div_flux(radius, l_of_j, S, dS, fix_in=None, fix_out=None, bc_in="field", bc_out="field"):
    """Divergence spectra (J*Nr, j fastest) of the flux vector with poloidal
    column S and radial-derivative column dS, fixed-field values fix_in /
    fix_out (J each, default zero) at the first and last radius; with
    bc_in / bc_out = "flux" that side has a fixed flux instead
    (cal_div_sph_in_fix_flux_2 / cal_div_sph_out_fix_flux_2,
    MHD_src/sph_MHD/cal_sph_exp_fixed_flux.f90:134-157, 253-276): the row takes
    the given flux (fix_in / fix_out) in place of the one-sided derivative."""
    r = np.asarray(radius, dtype=np.float64)
    nr, J = len(r), len(l_of_j)
    S = np.asarray(S).reshape(nr, J)
    dS = np.asarray(dS).reshape(nr, J)
    l = np.asarray(l_of_j)
    g3 = np.where(l == 0, 0.5, (l * (l + 1)).astype(np.float64))
    g3 = np.maximum(g3, 0.5)
    ar2 = (1.0 / r) ** 2
    d1, icb, cmb = fdm_coefs(r)
    fin = np.zeros(J) if fix_in is None else np.asarray(fix_in)
    fout = np.zeros(J) if fix_out is None else np.asarray(fix_out)
    out = np.zeros((nr, J))
    for k in range(1, nr - 1):
        d1s = d1[k, 0] * S[k - 1] + d1[k, 1] * S[k] + d1[k, 2] * S[k + 1]
        out[k] = (d1s - dS[k]) * g3 * ar2[k]
    d1s = fin if bc_in == "flux" else icb[0] * fin + icb[1] * S[1] + icb[2] * S[2]
    out[0] = (d1s - dS[0]) * g3 * ar2[0]
    d1s = fout if bc_out == "flux" else cmb[2] * S[nr - 3] + cmb[1] * S[nr - 2] + cmb[0] * fout
    out[nr - 1] = (d1s - dS[nr - 1]) * g3 * ar2[nr - 1]
    return out.reshape(-1)


def rot_uxb(radius, l_of_j, S, dS, T, bc_in="insulator", bc_out="insulator"):
    """Curl (pol, dpol/dr, tor) of the vector (S, dS/dr, T) with insulating
    boundaries, as const_sph_rotation_uxb
    (MHD_src/sph_MHD/const_sph_rotation.f90:167-187): interior rows
    cal_sph_nod_vect_w_div_rot2 (cal_sph_exp_rotation.f90:207-248)
        pol = T, dpol/dr = dT/dr (FDM), tor = -d(dS/dr)/dr (FDM) + g3 S / r^2,
    g3 = g_sph_rj(j,3) = l(l+1), 0 at l = 0: copy_sph_normalization_2_rj
    (CORE_src/SPH_SPECTR_src/schmidt_poly_on_rtm_grid.f90:117-140) applies no
    l = 0 override, unlike the rlm copy (:89-113);
    boundary rows cal_sph_nod_icb_ins_vp_rot2 (cal_sph_exp_nod_icb_ins.f90:135-160)
    and cal_sph_nod_cmb_ins_vp_rot2 (cal_sph_exp_nod_cmb_ins.f90:131-157):
        pol = T, dpol/dr = (l + 1) T / r (inner) or -l T / r (outer), tor = 0."""
    r = np.asarray(radius, dtype=np.float64)
    nr, J = len(r), len(l_of_j)
    S = np.asarray(S).reshape(nr, J)
    dS = np.asarray(dS).reshape(nr, J)
    T = np.asarray(T).reshape(nr, J)
    l = np.asarray(l_of_j).astype(np.float64)
    g3 = l * (l + 1.0)  # g_sph_rj(j,3): 0 at l = 0 in the rj copy
    ar1 = 1.0 / r
    ar2 = ar1 ** 2
    d1, _, _ = fdm_coefs(r)
    pol, dpol, tor = T.copy(), np.zeros((nr, J)), np.zeros((nr, J))
    for k in range(1, nr - 1):
        d1d = d1[k, 0] * dS[k - 1] + d1[k, 1] * dS[k] + d1[k, 2] * dS[k + 1]
        d1t = d1[k, 0] * T[k - 1] + d1[k, 1] * T[k] + d1[k, 2] * T[k + 1]
        dpol[k] = d1t
        tor[k] = -d1d + g3 * ar2[k] * S[k]
    dpol[0] = (l + 1.0) * ar1[0] * T[0]
    dpol[nr - 1] = -l * ar1[nr - 1] * T[nr - 1]
    # pseudo-vacuum (radial field): cal_sph_nod_icb_qvc_vp_rot2 /
    # cal_sph_nod_cmb_qvc_vp_rot2 (cal_sph_exp_nod_icb_qvac.f90:125-147,
    # cal_sph_exp_nod_cmb_qvac.f90:125-147): pol = T, dpol/dr = tor = 0
    if bc_in == "pseudo_vacuum":
        dpol[0] = 0.0
    if bc_out == "pseudo_vacuum":
        dpol[nr - 1] = 0.0
    return pol.reshape(-1), dpol.reshape(-1), tor.reshape(-1)


NON_SLIP, FREE_SLIP = "non_slip", "free_slip"


def velocity_bnd_coefs(radius, bc_icb=NON_SLIP, bc_cmb=NON_SLIP):
    """Boundary-row coefficients of the curl of a force: for each side,
    (s0, s1) of d2S/dr2 = s0 S(boundary) + s1 S(neighbour) and (t0, t1, t2) of
    dT/dr on the boundary node and its first and second neighbours."""
    r = np.asarray(radius, dtype=np.float64)
    _, icb, cmb = fdm_coefs(r)
    if bc_icb == NON_SLIP:
        dr = r[1] - r[0]
        # unknowns (S', S, S''), rows: S' fixed, S, S(kr + 1)
        m = inverse33([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [dr, 1.0, dr * dr / 2.0]])
        s_in, t_in = (m[2, 1], m[2, 2]), tuple(icb)
    elif bc_icb == FREE_SLIP:
        dr, r0 = r[1] - r[0], r[0]
        mvp = inverse33([[1.0, 0.0, 0.0], [1.0, -r0, 0.5 * r0 * r0], [1.0, dr, 0.5 * dr * dr]])
        mvt = inverse33([[1.0, 0.0, 0.0], [2.0, -r0, 0.0], [1.0, dr, 0.5 * dr * dr]])
        s_in, t_in = (mvp[2, 0], mvp[2, 2]), (mvt[1, 0], 0.0, 0.0)
    else:
        raise ValueError(bc_icb)
    if bc_cmb == NON_SLIP:
        dn = r[-1] - r[-2]
        m = inverse33([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [1.0, -dn, dn * dn / 2.0]])
        s_out, t_out = (m[2, 0], m[2, 2]), tuple(cmb)
    elif bc_cmb == FREE_SLIP:
        dn, r0 = r[-1] - r[-2], r[-1]
        mvp = inverse33([[1.0, 0.0, 0.0], [1.0, -r0, 0.5 * r0 * r0], [1.0, -dn, 0.5 * dn * dn]])
        mvt = inverse33([[1.0, 0.0, 0.0], [2.0, -r0, 0.0], [1.0, -dn, 0.5 * dn * dn]])
        s_out, t_out = (mvp[2, 0], mvp[2, 2]), (mvt[1, 0], 0.0, 0.0)
    else:
        raise ValueError(bc_cmb)
    return s_in, t_in, s_out, t_out


def rot_force(radius, l_of_j, S, dS, T, bc_icb=NON_SLIP, bc_cmb=NON_SLIP):
    """Curl (pol, dpol/dr, tor) of the force (S, dS/dr, T), as
    const_sph_force_rot2: interior rows as rot_uxb; boundary rows
        pol = T, dpol/dr = one-sided dT/dr, tor = -(d2S/dr2 - g3 S / r^2)
    with the velocity condition's coefficients (velocity_bnd_coefs)."""
    r = np.asarray(radius, dtype=np.float64)
    nr, J = len(r), len(l_of_j)
    pol, dpol, tor = (x.reshape(nr, J) for x in rot_uxb(r, l_of_j, S, dS, T))
    S = np.asarray(S).reshape(nr, J)
    T = np.asarray(T).reshape(nr, J)
    l = np.asarray(l_of_j).astype(np.float64)
    g3 = l * (l + 1.0)  # g_sph_rj(j,3): 0 at l = 0 in the rj copy
    ar2 = (1.0 / r) ** 2
    s_in, t_in, s_out, t_out = velocity_bnd_coefs(r, bc_icb, bc_cmb)
    d2s = s_in[0] * S[0] + s_in[1] * S[1]
    dpol[0] = t_in[0] * T[0] + t_in[1] * T[1] + t_in[2] * T[2]
    tor[0] = -(d2s - g3 * ar2[0] * S[0])
    d2s = s_out[1] * S[nr - 2] + s_out[0] * S[nr - 1]
    dpol[nr - 1] = t_out[2] * T[nr - 3] + t_out[1] * T[nr - 2] + t_out[0] * T[nr - 1]
    tor[nr - 1] = -(d2s - g3 * ar2[nr - 1] * S[nr - 1])
    return pol.reshape(-1), dpol.reshape(-1), tor.reshape(-1)


def div_force(radius, l_of_j, S, dS):
    """Divergence of a force (S, dS/dr), as const_sph_div_force: the fixed-field
    rows of div_flux with the boundary nodes' own S values."""
    nr = len(radius)
    S2 = np.asarray(S).reshape(nr, -1)
    return div_flux(radius, l_of_j, S, dS, fix_in=S2[0], fix_out=S2[-1])


def _d2_coefs(r):
    """Interior 3-point second derivative (offsets -1, 0, +1): row 2 of the
    inverse Taylor matrix, fdm(2) of copy_fdm2_nod_coefs_from_mat
    (CORE_src/SPH_SPECTR_src/t_fdm_coefs.f90:146-163)."""
    nr = len(r)
    d2 = np.zeros((nr, 3))
    for k in range(1, nr - 1):
        dp, dn = r[k + 1] - r[k], r[k] - r[k - 1]
        inv = inverse33(np.array([[1.0, 0.0, 0.0], [1.0, dp, 0.5 * dp * dp], [1.0, -dn, 0.5 * dn * dn]]))
        d2[k] = [inv[2, 2], inv[2, 0], inv[2, 1]]
    return d2


def _rot_field(radius, l_of_j, S, dS, T, bnd_rows):
    """Curl of a field (S, dS/dr, T): interior rows cal_sph_nod_vect_rot2
    (MHD_src/sph_MHD/cal_sph_exp_rotation.f90:157-203), pol = T, dpol/dr = d1 T,
    tor = -d2 S + g3 S / r^2; boundary rows from bnd_rows(k, S, T) -> (dpol, d2s)."""
    r = np.asarray(radius, dtype=np.float64)
    nr, J = len(r), len(l_of_j)
    S = np.asarray(S).reshape(nr, J)
    T = np.asarray(T).reshape(nr, J)
    l = np.asarray(l_of_j).astype(np.float64)
    g3 = l * (l + 1.0)
    ar2 = (1.0 / r) ** 2
    d1, _, _ = fdm_coefs(r)
    d2 = _d2_coefs(r)
    pol, dpol, tor = T.copy(), np.zeros((nr, J)), np.zeros((nr, J))
    for k in range(1, nr - 1):
        d2s = d2[k, 0] * S[k - 1] + d2[k, 1] * S[k] + d2[k, 2] * S[k + 1]
        dpol[k] = d1[k, 0] * T[k - 1] + d1[k, 1] * T[k] + d1[k, 2] * T[k + 1]
        tor[k] = -d2s + g3 * ar2[k] * S[k]
    for k in (0, nr - 1):
        dp, d2s = bnd_rows(k, S, T)
        dpol[k] = dp
        tor[k] = -(d2s - g3 * ar2[k] * S[k])
    return pol.reshape(-1), dpol.reshape(-1), tor.reshape(-1)


def vorticity(radius, l_of_j, S, dS, T, bc_icb=NON_SLIP, bc_cmb=NON_SLIP):
    """const_sph_vorticity (MHD_src/sph_MHD/const_sph_rotation.f90:111-137):
    interior rows of _rot_field, boundary rows of sel_bc_sph_vorticity (as
    rot_force)."""
    r = np.asarray(radius, dtype=np.float64)
    s_in, t_in, s_out, t_out = velocity_bnd_coefs(r, bc_icb, bc_cmb)
    nr = len(r)

    def rows(k, S, T):
        if k == 0:
            return t_in[0] * T[0] + t_in[1] * T[1] + t_in[2] * T[2], s_in[0] * S[0] + s_in[1] * S[1]
        return (t_out[2] * T[nr - 3] + t_out[1] * T[nr - 2] + t_out[0] * T[nr - 1],
                s_out[1] * S[nr - 2] + s_out[0] * S[nr - 1])
    return _rot_field(r, l_of_j, S, dS, T, rows)


INSULATOR, PSEUDO_VACUUM = "insulator", "pseudo_vacuum"


def current(radius, l_of_j, S, dS, T, bc_icb=INSULATOR, bc_cmb=INSULATOR):
    """const_sph_current (const_sph_rotation.f90:141-158) with sel_bc_sph_current
    (select_exp_magne_bc.f90:172-218): the non-slip coefficient rows, an
    insulator folding the potential field's dS/dr = (l+1) S / r (inner,
    cal_sph_nod_icb_ins_rot2) or -l S / r (outer, cal_sph_nod_cmb_ins_rot2)
    into the second derivative through the fixed derivative's coefficient
    (fdm2_fix_dr_ICB(-1,3), fdm2_fix_dr_CMB(1,3)); pseudo-vacuum rows keep
    dS/dr = 0 (cal_sph_nod_icb_qvc_rot2 / cal_sph_nod_cmb_qvc_rot2)."""
    r = np.asarray(radius, dtype=np.float64)
    nr = len(r)
    l = np.asarray(l_of_j).astype(np.float64)
    s_in, t_in, s_out, t_out = velocity_bnd_coefs(r, NON_SLIP, NON_SLIP)
    dr = r[1] - r[0]
    cdr_in = inverse33([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [dr, 1.0, dr * dr / 2.0]])[2, 0]
    dn = r[-1] - r[-2]
    cdr_out = inverse33([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [1.0, -dn, dn * dn / 2.0]])[2, 1]

    def rows(k, S, T):
        if k == 0:
            s0 = (l + 1.0) * (1.0 / r[0]) * cdr_in + s_in[0] if bc_icb == INSULATOR else s_in[0]
            return t_in[0] * T[0] + t_in[1] * T[1] + t_in[2] * T[2], s0 * S[0] + s_in[1] * S[1]
        s0 = s_out[0] - l * (1.0 / r[nr - 1]) * cdr_out if bc_cmb == INSULATOR else s_out[0]
        return (t_out[2] * T[nr - 3] + t_out[1] * T[nr - 2] + t_out[0] * T[nr - 1],
                s_out[1] * S[nr - 2] + s0 * S[nr - 1])
    return _rot_field(r, l_of_j, S, dS, T, rows)


def rot_buoyancy(radius, J, T, coef_t, C=None, coef_c=0.0):
    """cal_rot_buoyancy_sph_MHD / cal_rot_double_buoyancy_sph_MHD
    (MHD_src/sph_MHD/cal_rot_buoyancies_sph_MHD.f90:106-165): coef T r, or
    (coef_t T + coef_c C) r."""
    r = np.repeat(np.asarray(radius, dtype=np.float64), J)
    T = np.asarray(T)
    if C is None:
        return coef_t * T * r
    return (coef_t * T + coef_c * np.asarray(C)) * r
