"""Drop-in for planar_beads/fdtd2d_core.py: run_beads (full-domain method) and
save_results, with the time loop on the B200 engine.

Same signature, same physics setup (materials, sub-pixel bead, TE/TM
coefficients, CPML, VCSEL Huygens source), same schedule (step count, detector
windows, CW DFT over the last 8 periods, convergence extension, snapshots) and
the same result dictionary and output files as the reference
(fdtd2d_core.py:531-927, 2020-2049, 2085-2265).  Supported: method='full',
boundary='cpml', source_type='cw', no CAD, flat (not curved) geometry; other
methods raise NotImplementedError.
"""
import os
import pickle
import time

import numpy as np
import torch

from . import engine as E
from .geometry import Bead2D, Spec2D, Stack, air_path_um, build_2d
from .physics import C0, cornea_default, n_at

# module switches the reference's driver sets (fdtd2d_core.py:33-62)
KAPPA = {}
SRC_CORE_ONLY = False
LASER_POWER_MW = 20.0
TEAR_BUFFER = 10.0e-6
AIR_BUFFER = 5.0e-6
L_DEMO = 1.0e-3
T_MU = 0.5e-6
T_AQ = 3.5e-6
DET_LEN = 30e-6
N_G_FACTOR = 1.10
CW_TOL = 0.01
CW_MAX_EXTEND = 2.0
N_LIPID = 1.480


def _set_tear(stack, tear_buffer_um, dx_nm, cad=None):
    """The reference's run_beads preamble (fdtd2d_core.py:547-560): a custom stack
    deepens the domain below the core when the fixed buffer is too shallow; an
    explicit tear_buffer_um sets it.  The caller restores TEAR_BUFFER."""
    global TEAR_BUFFER
    if stack is not None and tear_buffer_um is None and cad is None:
        need = sum(float(Ly['t_um']) for Ly in stack) + 1.5 + 10 * dx_nm * 1e-3
        if need * 1e-6 > TEAR_BUFFER + 1e-12:
            tear_buffer_um = need
    if tear_buffer_um is not None:
        TEAR_BUFFER = float(tear_buffer_um) * 1e-6


def _guard_in_plane(i_in, src_ix, n_max, margin=5):
    lo = int(src_ix) + int(margin)
    return int(i_in) if i_in >= lo else min(lo, int(n_max) - 2)


def _legacy_stack(wg_n, t_wg_um, t_lip, n_lip, t_aq, n_aq, t_mu, n_mu, n_co, lossy, k):
    """Lipid / aqueous / mucin below the core on the cornea (fdtd2d_core.py:144-213)."""
    layers, thick = [], []
    for t, n, key in ((t_lip, n_lip, 'lip'), (t_aq, n_aq, 'aq'), (t_mu, n_mu, 'mu')):
        if key == 'lip' and t <= 1e-12:
            continue
        layers.append((t * 1e6, complex(n, k.get(key, 0.0)) if lossy else n))
        thick.append(t)
    return Stack(complex(wg_n, k.get('wg', 0.0)) if lossy else wg_n, t_wg_um, layers, n_co,
                 thick_m=thick, k_sub=k.get('co', 0.0) if lossy else 0.0, force_lossy=lossy)


def run_beads(wg_mat, bead_mat, bead_d_um, dx_nm=20.0, save_frames=True, n_snapshots=12,
              wg_thickness_um=5.0, lambda_nm=850.0, vcsel_waist=3.0, vcsel_tilt=0.0,
              vcsel_offset=0.0, source_type='cw', method='full',
              window_w_um=350.0, slide_um=150.0, place_bead=True, t_aqueous_um=None,
              t_mucin_um=None, t_lipid_um=0.0, input_gap_um=0.0, length_um=None,
              bead_x_um=None, bead_y_um=None, wg_n=None, bead_n=None, n_aqueous=None, n_mucin=None,
              n_cornea=None, n_lipid=None, polarization='s', curved=False, boundary='cpml',
              cad=None, pulse_cycles=30.0, pulse_tmax_fs=None, pulse_nfreq=None,
              pulse_dispersion=True, pulse_mode='fourier', n_aq_tear_offset=None,
              tear_buffer_um=None, stack=None):
    """2D TE/TM full-domain CW solve (fdtd2d_core.py:531-927) on the GPU engine;
    method='stitch' runs run_beads_stitched (fdtd2d_core.py:599-608)."""
    if method == 'stitch' and str(source_type).lower() != 'pulse':
        global TEAR_BUFFER
        old = TEAR_BUFFER
        if stack is not None and tear_buffer_um is None and cad is None:
            need = sum(float(L['t_um']) for L in stack) + 1.5 + 10 * dx_nm * 1e-3
            if need * 1e-6 > TEAR_BUFFER + 1e-12:
                tear_buffer_um = need
        if tear_buffer_um is not None:
            TEAR_BUFFER = float(tear_buffer_um) * 1e-6
        try:
            return run_beads_stitched(wg_mat, bead_mat, bead_d_um, dx_nm, save_frames, n_snapshots,
                                      wg_thickness_um, lambda_nm, vcsel_waist, vcsel_tilt, vcsel_offset,
                                      source_type, window_w_um, slide_um, place_bead, t_aqueous_um,
                                      t_mucin_um=t_mucin_um, t_lipid_um=t_lipid_um, input_gap_um=input_gap_um,
                                      length_um=length_um, bead_x_um=bead_x_um, bead_y_um=bead_y_um, wg_n=wg_n,
                                      bead_n=bead_n, n_aqueous=n_aqueous, n_mucin=n_mucin, n_cornea=n_cornea,
                                      n_lipid=n_lipid, polarization=polarization, curved=curved,
                                      boundary=boundary, cad=cad, stack=stack)
        finally:
            TEAR_BUFFER = old
    if method == 'stitch' and str(source_type).lower() == 'pulse':
        if pulse_mode == 'td':
            raise NotImplementedError("lens_sensor_b200.run_beads: the time-domain pulse stitch "
                                      "(pulse_mode='td') is not built; the Fourier stitch is")
        global_old = TEAR_BUFFER
        try:
            _set_tear(stack, tear_buffer_um, dx_nm, cad)
            return run_beads_stitched_pulse(
                wg_mat, bead_mat, bead_d_um, dx_nm, save_frames, n_snapshots, wg_thickness_um, lambda_nm,
                vcsel_waist, vcsel_tilt, vcsel_offset, window_w_um, slide_um, place_bead,
                t_aqueous_um=t_aqueous_um, t_mucin_um=t_mucin_um, t_lipid_um=t_lipid_um, input_gap_um=input_gap_um,
                length_um=length_um, bead_x_um=bead_x_um, bead_y_um=bead_y_um, wg_n=wg_n, bead_n=bead_n,
                n_aqueous=n_aqueous, n_mucin=n_mucin, n_cornea=n_cornea, n_lipid=n_lipid,
                polarization=polarization, curved=curved, boundary=boundary, cad=cad, pulse_cycles=pulse_cycles,
                pulse_tmax_fs=pulse_tmax_fs, pulse_nfreq=pulse_nfreq, pulse_dispersion=pulse_dispersion,
                n_aq_tear_offset=n_aq_tear_offset, stack=stack)
        finally:
            globals()['TEAR_BUFFER'] = global_old
    if method == 'sliding':
        global_old = TEAR_BUFFER
        try:
            _set_tear(stack, tear_buffer_um, dx_nm, cad)
            return run_beads_sliding(wg_mat, bead_mat, bead_d_um, dx_nm, save_frames, n_snapshots,
                                     wg_thickness_um, lambda_nm, vcsel_waist, vcsel_tilt, vcsel_offset,
                                     source_type, window_w_um, slide_um, place_bead, t_aqueous_um,
                                     t_mucin_um=t_mucin_um, t_lipid_um=t_lipid_um, input_gap_um=input_gap_um,
                                     length_um=length_um, bead_x_um=bead_x_um, bead_y_um=bead_y_um, wg_n=wg_n,
                                     bead_n=bead_n, n_aqueous=n_aqueous, n_mucin=n_mucin, n_cornea=n_cornea,
                                     n_lipid=n_lipid, polarization=polarization, curved=curved,
                                     boundary=boundary, pulse_cycles=pulse_cycles, cad=cad, stack=stack)
        finally:
            globals()['TEAR_BUFFER'] = global_old
    if method != 'full' or str(boundary).lower() != 'cpml' or source_type != 'cw' or cad is not None or curved:
        raise NotImplementedError(f'lens_sensor_b200.run_beads: method={method!r} boundary={boundary!r} '
                                  f'source_type={source_type!r} cad={cad is not None} curved={curved}: '
                                  f'only the full-domain CPML CW path runs on the B200 engine')
    if stack is not None and tear_buffer_um is None:
        need = sum(float(L['t_um']) for L in stack) + 1.5 + 10 * dx_nm * 1e-3
        if need * 1e-6 > TEAR_BUFFER + 1e-12:
            tear_buffer_um = need
    tear_m = float(tear_buffer_um) * 1e-6 if tear_buffer_um is not None else TEAR_BUFFER
    pol = 'p' if str(polarization).lower() in ('p', 'tm') else 's'
    t_aq_um = t_aqueous_um if t_aqueous_um is not None else T_AQ * 1e6
    t_total = time.time()
    wg_n = wg_n if wg_n is not None else n_at(wg_mat, lambda_nm)
    bead_n = bead_n if bead_n is not None else n_at(bead_mat, lambda_nm)
    n_aq_l = n_aqueous if n_aqueous is not None else n_at('aqueous', lambda_nm)
    n_mu_l = n_mucin if n_mucin is not None else n_at('mucin', lambda_nm)
    n_co_l = n_cornea if n_cornea is not None else cornea_default(lambda_nm)
    n_lip_l = n_lipid if n_lipid is not None else n_at('lipid', lambda_nm)
    L = (length_um * 1e-6) if length_um is not None else L_DEMO
    L_um = L * 1e6
    bx_um = bead_x_um if bead_x_um is not None else L_um / 2.0
    T_WG = wg_thickness_um * 1e-6
    label = f'WG-{wg_mat}_Bead-{bead_mat}_d{bead_d_um:g}_L{lambda_nm:g}' + ('' if place_bead else '_ref')
    dx = dx_nm * 1e-9
    NPML = 10
    src_ix = NPML + 2
    vd = float(input_gap_um or 0.0)
    air = air_path_um(vd, dx * 1e6)
    x_facet_um = src_ix * dx * 1e6 + air
    H_total = T_WG + AIR_BUFFER + tear_m
    Nx, Ny = int(round(L / dx)), int(round(H_total / dx))
    k = dict(KAPPA or {})
    if stack is None:
        lossy = any(v > 0 for v in k.values())
        t_mu = (t_mucin_um * 1e-6) if t_mucin_um is not None else T_MU
        st = _legacy_stack(wg_n, wg_thickness_um, (t_lipid_um or 0.0) * 1e-6, n_lip_l, t_aq_um * 1e-6,
                           n_aq_l, t_mu, n_mu_l, n_co_l, lossy, k)
    else:
        lossy = any(v > 0 for v in k.values()) or any(complex(Ly['n']).imag > 0 for Ly in stack)
        st = Stack(complex(wg_n, k.get('wg', 0.0)) if lossy else wg_n, wg_thickness_um,
                   [(float(Ly['t_um']), complex(Ly['n'])) for Ly in stack], n_co_l,
                   k_sub=k.get('co', 0.0) if lossy else 0.0, force_lossy=lossy)
    bead = None
    if place_bead and bead_d_um:
        bead = Bead2D(bx_um, bead_d_um, complex(bead_n, k.get('bead', 0.0)) if lossy else bead_n, bead_y_um)
    sp = Spec2D(pol, Nx, Ny, dx, st, tear_m, bead, npml=NPML, lam_nm=lambda_nm, waist_um=vcsel_waist,
                length_m=L, vcsel_distance_um=vd, vcsel_offset_um=vcsel_offset, vcsel_tilt_deg=vcsel_tilt,
                src_core_only=SRC_CORE_ONLY)
    geo = build_2d(sp)
    dt, f0 = sp.dt, sp.f0
    coef = {q: geo[q] for q in ('ce_e', 'ce_h', 'ca_x', 'ca_y', 'da_x', 'da_y') if q in geo}
    g = E.Grid2D(pol, Nx, Ny, dx, dt, coef, geo['cx'], geo['cy'], geo['src'])
    sigma_t = 4 / (2 * np.pi * f0)
    steps_total = int((6 * sigma_t + 2 * L * N_G_FACTOR * float(np.real(wg_n)) / C0) / dt)
    steps_max = int(CW_MAX_EXTEND * steps_total)
    snap_every = max(1, steps_total // n_snapshots)
    iy_lo, iy_hi = int(round((0.0 + tear_m) / dx)), int(round((T_WG + tear_m) / dx))
    hw = max(1, int(round(min(DET_LEN / 2, 0.05 * L_um * 1e-6) / dx)))

    def xwin(xu):
        c = int(round(xu * 1e-6 / dx))
        return max(0, c - hw), min(Nx, c + hw)
    ixin0, ixin1 = xwin(0.1 * L_um)
    ixout0, ixout1 = xwin(0.9 * L_um)
    ci = (ixin0 + ixin1) // 2
    sh = _guard_in_plane(ci, max(src_ix, int(round(x_facet_um / (dx * 1e6)))), Nx) - ci
    ixin0, ixin1 = ixin0 + sh, min(Nx, ixin1 + sh)
    planes = {'in': max(1, (ixin0 + ixin1) // 2), 'out': max(1, (ixout0 + ixout1) // 2),
              'src_up': src_ix - 1, 'src_dn': src_ix + 3}
    omega = 2 * np.pi * f0
    steps_per_T = max(4, int(round((1.0 / f0) / dt)))
    n_acc = 8 * steps_per_T
    n_avg0 = steps_total // 2
    tab = E.StepTable(0, steps_max + n_acc, dt, geo['src']['omega'], omega, E.cw_envelope(f0))
    ep = E.Epi2D(g, boxes=[(ixin0, ixin1, iy_lo, iy_hi), (ixout0, ixout1, iy_lo, iy_hi)],
                 dft=(steps_total - n_acc, steps_total), dft_ex=(pol == 'p'),
                 prev=(steps_total - 2 * n_acc, steps_total - n_acc), iavg_n0=n_avg0, planes=planes)
    y0_m = -tear_m
    frames, mm_path, ez_mm = [], None, None
    safe = ''.join(c if (c.isalnum() or c in '-_.') else '_' for c in label)
    if save_frames:
        os.makedirs('results', exist_ok=True)
        mm_path = os.path.join('results', f'_stream_beads_{safe}_full.npy')
        ez_mm = np.lib.format.open_memmap(mm_path, mode='w+', dtype=np.float32,
                                          shape=(max(1, n_snapshots + 2), Nx, Ny))
    t_start = time.time()
    n, k_fr, cw_rel_change, nacc_prev = 0, 0, float('nan'), n_acc
    while n < steps_total:
        nxt = min(steps_total, ((n // snap_every) + 1) * snap_every)
        g.step(tab, n, nxt - n, ep)
        n = nxt
        if save_frames and n % snap_every == 0 and k_fr < ez_mm.shape[0]:
            ez_mm[k_fr] = _field_2d(g)
            frames.append({'x_start': 0.0, 'x_end': L_um, 'y_start': y0_m * 1e6,
                           'y_end': (y0_m + H_total) * 1e6, 'slide_i': 0, 'step': n,
                           'time': time.time() - t_start})
            k_fr += 1
        if n == steps_total:
            a = ep.phasor() / n_acc
            b = ep.phasor('prev') / nacc_prev
            cw_rel_change = float(torch.linalg.norm(a - b)) / max(float(torch.linalg.norm(a)), 1e-30)
            if cw_rel_change > CW_TOL and steps_total + n_acc <= steps_max:
                ep.restart_dft((steps_total, steps_total + n_acc))
                nacc_prev = n_acc
                steps_total += n_acc
    if ez_mm is not None:
        ez_mm.flush()
        del ez_mm
    Ecw = ((2.0 / n_acc) * ep.phasor()).cpu().numpy()
    cw_path, cw_frames = None, []
    nfr_cw = max(1, n_snapshots)
    if save_frames:
        cw_path = os.path.join('results', f'_stream_beads_{safe}_full_cw.npy')
        cw_mm = np.lib.format.open_memmap(cw_path, mode='w+', dtype=np.float32, shape=(nfr_cw, Nx, Ny))
        for q in range(nfr_cw):
            tk = (q / nfr_cw) * (1.0 / f0)
            cw_mm[q] = np.real(Ecw * np.exp(1j * omega * tk)).astype(np.float32)
            cw_frames.append({'x_start': 0.0, 'x_end': L_um, 'y_start': y0_m * 1e6,
                              'y_end': (y0_m + H_total) * 1e6, 'slide_i': 0, 'step': q, 'time': tk})
        cw_mm.flush()
        del cw_mm
    box = ep.box_acc.double().cpu().numpy()
    P_in, P_out = float(box[0]) * dx * dx, float(box[1]) * dx * dx
    Tr_I = P_out / max(P_in, 1e-30)
    S_in, S_out = ep.flux('in', n_acc), ep.flux('out', n_acc)
    Tr, tr_def, p_si = Tr_I, 'intensity', S_in * dx
    if abs(S_in) > 0:
        Tr, tr_def = S_out / S_in, 'poynting'
    res = _result_dict(label, P_in, P_out, Tr, frames, time.time() - t_total, bead_d_um, wg_mat, bead_mat,
                       wg_n, bead_n, wg_thickness_um, lambda_nm, vcsel_waist, vcsel_tilt, vcsel_offset,
                       source_type, 'full', place_bead, n_aq_l, n_mu_l, n_co_l, mm_path, t_aq_um,
                       t_mucin_um, t_lipid_um, bx_um, x_facet_um, L_um, pol, stack, n_lip_l)
    res['Iavg'] = (ep.iavg[:, :Ny].cpu().numpy() / max(1, steps_total - n_avg0))
    res['cw_frames'] = cw_frames
    res['cw_frames_memmap'] = cw_path
    res['cw_rel_change'] = cw_rel_change
    if pol == 'p':
        res['Ex_cw_amp'] = ((2.0 / n_acc) * ep.phasor('dft_ex')).cpu().numpy()
    res['transmission_intensity'] = Tr_I
    res['transmission_def'] = tr_def
    res['steps_total'] = steps_total
    res['p_in_si'] = p_si
    res['p_in_unit'] = 'W/m'
    up, dn = ep.flux('src_up', n_acc), ep.flux('src_dn', n_acc)
    p_emit, p_refl = (dn - up) * dx, -up * dx
    res.update(laser_power_mw=LASER_POWER_MW, vcsel_distance_um=vd, vcsel_air_um=float(air),
               vcsel_waist_um=float(vcsel_waist), x_facet_um=float(x_facet_um), p_src_si=p_emit)
    if p_emit and p_emit > 0:
        res['coupling_efficiency'] = p_si / p_emit
        res['facet_reflection'] = p_refl / p_emit
    res['view_primary'] = 'transient'
    res['Ecw'] = Ecw
    return res


def _stack_2d(wg_n, wg_thickness_um, t_lipid_um, n_lip, t_aq_um, n_aq, t_mucin_um, n_mu, n_co, stack):
    """Layer stack and loss switch of run_beads (fdtd2d_core.py:144-213)."""
    k = dict(KAPPA or {})
    if stack is None:
        lossy = any(v > 0 for v in k.values())
        t_mu = (t_mucin_um * 1e-6) if t_mucin_um is not None else T_MU
        st = _legacy_stack(wg_n, wg_thickness_um, (t_lipid_um or 0.0) * 1e-6, n_lip, t_aq_um * 1e-6,
                           n_aq, t_mu, n_mu, n_co, lossy, k)
    else:
        lossy = any(v > 0 for v in k.values()) or any(complex(Ly['n']).imag > 0 for Ly in stack)
        st = Stack(complex(wg_n, k.get('wg', 0.0)) if lossy else wg_n, wg_thickness_um,
                   [(float(Ly['t_um']), complex(Ly['n'])) for Ly in stack], n_co,
                   k_sub=k.get('co', 0.0) if lossy else 0.0, force_lossy=lossy)
    return st, lossy, k


def _node2d(F):
    """(nx, ny-1) -> (nx, ny) onto the nodes (fdtd2d_core.py:1497-1500)."""
    o = np.zeros((F.shape[0], F.shape[1] + 1), dtype=np.float32)
    o[:, 1:-1] = 0.5 * (F[:, :-1] + F[:, 1:])
    o[:, 0], o[:, -1] = F[:, 0], F[:, -1]
    return o


def run_beads_stitched(wg_mat, bead_mat, bead_d_um, dx_nm, save_frames, n_snapshots,
                       wg_thickness_um, lambda_nm, vcsel_waist, vcsel_tilt,
                       vcsel_offset, source_type, window_w_um, slide_um, place_bead=True,
                       t_aqueous_um=None, t_mucin_um=None, t_lipid_um=0.0, input_gap_um=0.0,
                       length_um=None, bead_x_um=None, bead_y_um=None, wg_n=None, bead_n=None,
                       n_aqueous=None, n_mucin=None, n_cornea=None, n_lipid=None,
                       polarization='s', curved=False, boundary='cpml', cad=None,
                       return_efull=False, stack=None):
    """2D CW solve by domain decomposition along x (fdtd2d_core.py:1197-1583).

    Windows of window_w_um slide by slide_um; each runs steps_win steps on the
    engine.  Window 0 carries the VCSEL; window w > 0 is driven on its first
    O = window - slide rows by the previous window's complex amplitude of the
    driven component (TE Ez, TM Ey) with a cosine taper; the amplitude stays on
    the device between windows.  Interior window ends get a CPML in an absorber
    extension that is not assembled.  The assembled CW amplitude gives the CW
    phase frames, the detector powers and (TM) <|E|^2> and the Ex amplitude.
    Supported: boundary='cpml', no CAD, flat geometry."""
    if str(boundary or 'cpml').lower() != 'cpml' or cad is not None or curved:
        raise NotImplementedError(f'lens_sensor_b200.run_beads_stitched: boundary={boundary!r} '
                                  f'cad={cad is not None} curved={curved}: only the CPML stitch runs on '
                                  f'the B200 engine')
    pol = 'p' if str(polarization).lower() in ('p', 'tm') else 's'
    t_total = time.time()
    t_aq_um = t_aqueous_um if t_aqueous_um is not None else T_AQ * 1e6
    wg_n = wg_n if wg_n is not None else n_at(wg_mat, lambda_nm)
    bead_n = bead_n if bead_n is not None else n_at(bead_mat, lambda_nm)
    n_aq_l = n_aqueous if n_aqueous is not None else n_at('aqueous', lambda_nm)
    n_mu_l = n_mucin if n_mucin is not None else n_at('mucin', lambda_nm)
    n_co_l = n_cornea if n_cornea is not None else cornea_default(lambda_nm)
    n_lip_l = n_lipid if n_lipid is not None else n_at('lipid', lambda_nm)
    L = (length_um * 1e-6) if length_um is not None else L_DEMO
    L_um = L * 1e6
    T_WG = wg_thickness_um * 1e-6
    LAM = lambda_nm * 1e-9
    bx_um = bead_x_um if bead_x_um is not None else L_um / 2.0
    label = f'WG-{wg_mat}_Bead-{bead_mat}_d{bead_d_um:g}_L{lambda_nm:g}' + ('' if place_bead else '_ref')
    dx = dx_nm * 1e-9
    dt = 0.5 * dx / (C0 * np.sqrt(2))
    NPML = 10
    src_ix = NPML + 2
    vd = float(input_gap_um or 0.0)
    air = air_path_um(vd, dx * 1e6)
    x_facet_um = src_ix * dx * 1e6 + air
    tear_m = TEAR_BUFFER
    y0_m = -tear_m
    H_total = T_WG + AIR_BUFFER + tear_m
    Ny = int(round(H_total / dx))
    Nx_win = int(round(window_w_um * 1e-6 / dx))
    S = int(round(slide_um * 1e-6 / dx))
    O = Nx_win - S
    Nx_full = int(round(L / dx))
    if O < 8:
        O = max(O, 1)
    f0 = C0 / LAM
    omega = 2 * np.pi * f0
    sigma_t = 4 / (2 * np.pi * f0)
    transit = window_w_um * 1e-6 * N_G_FACTOR * wg_n / C0
    steps_win = int(3.0 * transit / dt) + 400
    steps_per_T = max(4, int(round((1.0 / f0) / dt)))
    n_acc = steps_per_T * 8
    n_win = (int(np.ceil((Nx_full - Nx_win) / S)) + 1) if Nx_full > Nx_win else 1
    n_w0 = max(0, steps_win - n_acc)
    acc_n = steps_win - n_w0
    st, lossy, k = _stack_2d(wg_n, wg_thickness_um, t_lipid_um, n_lip_l, t_aq_um, n_aq_l, t_mucin_um, n_mu_l,
                             n_co_l, stack)
    bead = None
    if place_bead and bead_d_um:
        bead = Bead2D(bx_um, bead_d_um, complex(bead_n, k.get('bead', 0.0)) if lossy else bead_n, bead_y_um)

    def gx0(w):                          # the last window ends flush with the domain
        return min(w * S, max(Nx_full - Nx_win, 0))
    EXT = NPML + 4
    len_mat = L_um + EXT * dx * 1e6      # the core runs on into the absorber extension
    iy_lo, iy_hi = int(round((0.0 + tear_m) / dx)), int(round((T_WG + tear_m) / dx))
    ix_in, ix_out = int(round(0.1 * Nx_full)), int(round(0.9 * Nx_full))
    ix_in = _guard_in_plane(ix_in, max(src_ix, int(round(x_facet_um / (dx * 1e6)))), Nx_full)
    plan = []
    for w in range(n_win):
        g0, last = gx0(w), w == n_win - 1
        glo = 0 if w == 0 else g0 + O
        ghi = min(g0 + Nx_win, Nx_full)
        fpl = {q: g - g0 for q, g in (('in', ix_in), ('out', ix_out)) if glo <= g < ghi and g - g0 >= 1}
        if w == 0:
            fpl.update(src_up=src_ix - 1, src_dn=src_ix + 3)
        plan.append((g0, last, fpl))
    if not all(any(q in p[2] for p in plan) for q in ('in', 'out')):
        raise NotImplementedError('lens_sensor_b200.run_beads_stitched: a detector plane falls on a window '
                                  'start (no overlap); the E-only flux estimate is not built')
    Nyc = Ny - 1 if pol == 'p' else Ny
    Efull = np.zeros((Nx_full, Nyc), dtype=np.complex64)
    safe = ''.join(c if (c.isalnum() or c in '-_.') else '_' for c in label)
    ExI_full = ExA_full = None
    if pol == 'p':
        os.makedirs('results', exist_ok=True)
        tag = f'{os.getpid()}_{int(time.time() * 1000)}'
        ExI_full = np.lib.format.open_memmap(os.path.join('results', f'_stream_beads_{safe}_stitch_Iavg_{tag}.npy'),
                                             mode='w+', dtype=np.float32, shape=(Nx_full, Ny))
        ExA_full = np.lib.format.open_memmap(os.path.join('results', f'_stream_beads_{safe}_stitch_ExA_{tag}.npy'),
                                             mode='w+', dtype=np.complex64, shape=(Nx_full, Ny))
    wtap = (0.5 * (1.0 + np.cos(np.pi * np.arange(O) / max(O - 1, 1)))).astype(np.float32)
    # per-step FP64 drive values: the envelope and e^{i w t} as the reference forms them
    tq = np.arange(steps_win) * dt
    env_t = np.array([float(1 - np.exp(-((t / (2 * sigma_t)) ** 2))) for t in tq])
    ph_t = np.exp(1j * omega * tq)
    flux = FluxSum2D(E)
    hand = None
    geo0 = None
    tab = None
    sc = torch.tensor(2.0 / max(acc_n, 1), dtype=torch.float32)
    for w, (g0, last, fpl) in enumerate(plan):
        Nxw = Nx_win + (0 if last else EXT)
        sp = Spec2D(pol, Nxw, Ny, dx, st, tear_m, bead, npml=NPML, lam_nm=lambda_nm, waist_um=vcsel_waist,
                    length_m=len_mat * 1e-6, vcsel_distance_um=vd, vcsel_offset_um=vcsel_offset,
                    vcsel_tilt_deg=vcsel_tilt, src_core_only=SRC_CORE_ONLY, x_start_um=g0 * dx * 1e6,
                    npml_x=(NPML if w == 0 else 0, NPML))
        geo = build_2d(sp)
        if w == 0:
            geo0 = geo
            tab = E.StepTable(0, steps_win, dt, geo['src']['omega'], omega, E.cw_envelope(f0))
        coef = {q: geo[q] for q in ('ce_e', 'ce_h', 'ca_x', 'ca_y', 'da_x', 'da_y') if q in geo}
        grid = E.Grid2D(pol, Nxw, Ny, dx, dt, coef, geo['cx'], geo['cy'], geo['src'] if w == 0 else None,
                        pec=(1 if w == 0 else 0, 1, 1, 1))
        ep = E.Epi2D(grid, dft=(n_w0, steps_win), dft_ex=(pol == 'p'), planes=fpl, dft_raw=(pol == 'p'),
                     ex2=(pol == 'p'))
        drive = (E.Drive2D(grid, hand, wtap, env_t, ph_t.real, ph_t.imag)
                 if (w > 0 and hand is not None) else None)
        grid.step(tab, 0, steps_win, ep, drive=drive)
        a = ep.phasor('dft_raw' if pol == 'p' else 'dft', kind='stitch')
        s_ = sc.to(a.device)
        Ew_d = torch.complex(a.real.float() * s_, a.imag.float() * s_)
        if not last:
            off = gx0(w + 1) - g0
            hand = Ew_d[off:off + O]
        for q in fpl:
            flux.add(q, ep.plane_dft(q), acc_n)
        l_lo, g_lo = (0, 0) if w == 0 else (O, g0 + O)
        g_hi = min(g0 + Nx_win, Nx_full)
        l_hi = l_lo + (g_hi - g_lo)
        if g_hi > g_lo:
            Efull[g_lo:g_hi] = Ew_d[l_lo:l_hi].cpu().numpy()
            if ExI_full is not None:
                ExI_full[g_lo:g_hi] = ep.ex2[l_lo:l_hi, :Ny].cpu().numpy() / max(acc_n, 1)
                xa = ep.phasor('dft_ex', kind='stitch')[l_lo:l_hi]
                ExA_full[g_lo:g_hi] = torch.complex(xa.real.float() * s_, xa.imag.float() * s_).cpu().numpy()
        del grid, ep, drive
    total_time = time.time() - t_total
    frames, mm_path = [], None
    nfr = max(1, n_snapshots)
    if save_frames:
        os.makedirs('results', exist_ok=True)
        mm_path = os.path.join('results', f'_stream_beads_{safe}_stitch.npy')
        ez_mm = np.lib.format.open_memmap(mm_path, mode='w+', dtype=np.float32, shape=(nfr, Nx_full, Ny))
        for q in range(nfr):
            tk = (q / nfr) * (1.0 / f0)
            fr = np.real(Efull * np.exp(1j * omega * tk)).astype(np.float32)
            ez_mm[q] = _node2d(fr) if pol == 'p' else fr
            frames.append({'x_start': 0.0, 'x_end': L_um, 'y_start': y0_m * 1e6,
                           'y_end': (y0_m + H_total) * 1e6, 'slide_i': 0, 'step': q, 'time': tk})
        ez_mm.flush()
        del ez_mm
    # detector powers from the assembled amplitude (fdtd2d_core.py:1506-1519)
    P_in = float(np.sum(np.abs(Efull[ix_in, iy_lo:iy_hi]) ** 2))
    P_out = float(np.sum(np.abs(Efull[ix_out, iy_lo:iy_hi]) ** 2))
    if ExI_full is not None:
        P_in += 2.0 * float(np.sum(ExI_full[ix_in, iy_lo:iy_hi]))
        P_out += 2.0 * float(np.sum(ExI_full[ix_out, iy_lo:iy_hi]))
        for x0 in range(0, Nx_full, 4096):
            x1 = min(x0 + 4096, Nx_full)
            s2 = 0.5 * np.abs(Efull[x0:x1]) ** 2
            ey2 = np.empty((x1 - x0, Ny), dtype=np.float32)
            ey2[:, 1:-1] = 0.5 * (s2[:, :-1] + s2[:, 1:])
            ey2[:, 0], ey2[:, -1] = s2[:, 0], s2[:, -1]
            ExI_full[x0:x1] += ey2
        ExI_full.flush()
    Tr_I = P_out / max(P_in, 1e-30)
    S_in, S_out = flux.flux('in'), flux.flux('out')
    p_si = S_in * dx
    Tr = S_out / S_in if abs(S_in) > 0 else Tr_I
    res = _result_dict(label, P_in, P_out, Tr, frames, total_time, bead_d_um, wg_mat, bead_mat, wg_n, bead_n,
                       wg_thickness_um, lambda_nm, vcsel_waist, vcsel_tilt, vcsel_offset, source_type, 'stitch',
                       place_bead, n_aq_l, n_mu_l, n_co_l, mm_path, t_aq_um, t_mucin_um, t_lipid_um, bx_um,
                       x_facet_um, L_um, pol, stack, n_lip_l)
    res['transmission_intensity'] = Tr_I
    res['transmission_def'] = 'poynting'
    res['view_primary'] = 'cw'
    res['cw_only'] = True
    res['p_in_si'] = p_si
    res['p_in_unit'] = 'W/m'
    ok = flux.has('src_up') and flux.has('src_dn')
    p_emit = (flux.flux('src_dn') - flux.flux('src_up')) * dx if ok else None
    p_refl = -flux.flux('src_up') * dx if ok else None
    res.update(laser_power_mw=LASER_POWER_MW, vcsel_distance_um=vd, vcsel_air_um=float(geo0['src']['air_um']),
               vcsel_waist_um=float(vcsel_waist), x_facet_um=float(x_facet_um), p_src_si=p_emit)
    if p_emit and p_emit > 0:
        res['coupling_efficiency'] = (p_si / p_emit) if p_si is not None else float('nan')
        res['facet_reflection'] = (p_refl / p_emit) if p_refl is not None else float('nan')
    if ExI_full is not None:
        res['Iavg'] = ExI_full
    if ExA_full is not None:
        ExA_full.flush()
        res['Ex_cw_amp'] = ExA_full
    if return_efull:
        res['Efull'] = Efull
    return res


def stack_at_lambda(stack, lam_nm):
    """The stack at another wavelength (fdtd2d_core.py:83-95): a layer that names
    its material takes that material's n at lam_nm and keeps its absorption;
    layers given by number stay as they are."""
    if stack is None:
        return None
    out = []
    for Ly in stack:
        q = dict(Ly)
        if q.get('mat'):
            nc = complex(n_at(q['mat'], lam_nm), complex(q['n']).imag)
            q['n'], q['kappa'] = nc, nc.imag
        out.append(q)
    return out


def run_beads_stitched_pulse(wg_mat, bead_mat, bead_d_um, dx_nm, save_frames, n_snapshots,
                             wg_thickness_um, lambda_nm, vcsel_waist, vcsel_tilt, vcsel_offset,
                             window_w_um, slide_um, place_bead, pulse_cycles=30.0,
                             pulse_tmax_fs=None, pulse_nfreq=None, pulse_dispersion=True,
                             cad=None, t_eval_s=None, n_aq_tear_offset=None, stack=None, **kw):
    """Transient 2D stitch by Fourier synthesis (fdtd2d_core.py:1866-2017).

    The source pulse exp(-((t - 3s)/s)^2) sin(w0 t), s = pulse_cycles / f0, is
    split into frequencies w_k = w0 + k dw inside |w - w0| < 5.26 / s (the band
    where its spectrum exceeds 1e-3 of the peak), dw = 2 pi / (1.6 t_max) or set
    by pulse_nfreq.  Every w_k runs a CW stitch on the engine (materials at
    lambda_k unless pulse_dispersion is off); its assembled amplitude E_k answers
    sin(w t) = Re(-i e^{iwt}), so the field at t is
    (1/pi) Re sum_k i E_k S(w_k) e^{i w_k t} dw with
    S(w) = (G(w - w0) - G(w + w0)) / 2i, G(v) = sqrt(pi) s e^{-(v s)^2/4} e^{-i v tc}.
    The time frames are summed frequency by frequency on the device (one FP32
    accumulator per frame); the CW set of the centre frequency and the
    transmission spectrum come with the result.  No CAD."""
    if cad is not None:
        raise NotImplementedError('lens_sensor_b200.run_beads_stitched_pulse: CAD geometry is not built')
    t_total = time.time()
    f0 = C0 / (lambda_nm * 1e-9)
    w0 = 2 * np.pi * f0
    s_p = pulse_cycles / f0
    tc = 3 * s_p
    pol = 'p' if str(kw.get('polarization', 's')).lower() in ('p', 'tm') else 's'
    L_um = kw.get('length_um') or L_DEMO * 1e6
    n_core = kw.get('wg_n') or n_at(wg_mat, lambda_nm)
    y0_um, y1_um = -TEAR_BUFFER * 1e6, (wg_thickness_um * 1e-6 + AIR_BUFFER) * 1e6
    t_max = (pulse_tmax_fs * 1e-15) if pulse_tmax_fs else tc + 3 * s_p + L_um * 1e-6 * n_core * 1.15 / C0
    half = 5.26 / s_p
    dw = 2 * half / max(int(pulse_nfreq) - 1, 1) if pulse_nfreq else 2 * np.pi / (1.6 * t_max)
    m = int(np.ceil(half / dw))
    w_k = w0 + np.arange(-m, m + 1) * dw
    w_k = w_k[w_k > 0]
    lam_k = 2 * np.pi * C0 / w_k * 1e9
    G = lambda v: np.sqrt(np.pi) * s_p * np.exp(-(v * s_p) ** 2 / 4.0) * np.exp(-1j * v * tc)
    S_k = (G(w_k - w0) - G(w_k + w0)) / (2j)
    fixed = {}
    if not pulse_dispersion:           # every index held at lambda0
        fixed = dict(wg_n=kw.get('wg_n') or n_at(wg_mat, lambda_nm),
                     bead_n=kw.get('bead_n') or n_at(bead_mat, lambda_nm),
                     n_aqueous=kw.get('n_aqueous') or n_at('aqueous', lambda_nm),
                     n_mucin=kw.get('n_mucin') or n_at('mucin', lambda_nm),
                     n_cornea=kw.get('n_cornea') or cornea_default(lambda_nm),
                     n_lipid=kw.get('n_lipid') or n_at('lipid', lambda_nm))
    rest = {q: v for q, v in kw.items() if q not in fixed}
    tear_disp = pulse_dispersion and n_aq_tear_offset is not None
    n_t = max(int(n_snapshots), 24)
    t_j = np.linspace(0.0, t_max, n_t)
    if t_eval_s is not None:
        t_j = np.asarray(t_eval_s, dtype=np.float64)
        n_t = len(t_j)
    label = f'WG-{wg_mat}_Bead-{bead_mat}_d{bead_d_um:g}_L{lambda_nm:g}' + ('' if place_bead else '_ref')
    safe = ''.join(c if (c.isalnum() or c in '-_.') else '_' for c in label)
    dev = torch.device('cuda') if torch.cuda.is_available() else torch.device('cpu')
    acc, spec_T, spec_P = None, [], []
    k_c = int(np.argmin(np.abs(w_k - w0)))
    r_c = E_c = None
    for k, (wk, lk, Sk) in enumerate(zip(w_k, lam_k, S_k)):
        kwk = dict(rest)
        if tear_disp:
            kwk['n_aqueous'] = n_at('aqueous', float(lk)) + float(n_aq_tear_offset)
        stk = stack_at_lambda(stack, float(lk)) if (stack is not None and pulse_dispersion) else stack
        r = run_beads_stitched(wg_mat, bead_mat, bead_d_um, dx_nm, False, 4, wg_thickness_um, float(lk),
                               vcsel_waist, vcsel_tilt, vcsel_offset, 'cw', window_w_um, slide_um, place_bead,
                               cad=None, return_efull=True, stack=stk, **fixed, **kwk)
        Ek = np.asarray(r.pop('Efull'))
        if pol == 'p':                 # Ey (nx, ny-1) onto the nodes (nx, ny)
            En = np.empty((Ek.shape[0], Ek.shape[1] + 1), dtype=np.complex64)
            En[:, 1:-1] = 0.5 * (Ek[:, :-1] + Ek[:, 1:])
            En[:, 0], En[:, -1] = Ek[:, 0], Ek[:, -1]
            Ek = En
        if acc is None:
            acc = torch.zeros((n_t,) + Ek.shape, dtype=torch.float32, device=dev)
        # i E_k S(w_k) dw / pi, then its real part at every frame time
        c = (torch.from_numpy(Ek).to(dev) * 1j).to(torch.complex128) * complex(Sk * dw / np.pi)
        for j, tj in enumerate(t_j):
            acc[j] += torch.real(c * complex(np.exp(1j * wk * tj))).to(torch.float32)
        spec_T.append(float(r['transmission']))
        spec_P.append(float(r['P_out']))
        if k == k_c:
            r_c, E_c = r, Ek
    os.makedirs('results', exist_ok=True)
    mm_path = os.path.join('results', f'_stream_beads_{safe}_pulse_{os.getpid()}.npy')
    fr_mm = np.lib.format.open_memmap(mm_path, mode='w+', dtype=np.float32, shape=tuple(acc.shape))
    for j in range(n_t):
        fr_mm[j] = acc[j].cpu().numpy()
    fr_mm.flush()
    del fr_mm, acc
    frames = [{'x_start': 0.0, 'x_end': L_um, 'y_start': y0_um, 'y_end': y1_um, 'slide_i': 0, 'step': j,
               'time': float(tj)} for j, tj in enumerate(t_j)]
    # the steady set at the centre frequency (the analyzer's second view)
    cw_path = os.path.join('results', f'_stream_beads_{safe}_pulse_cw_{os.getpid()}.npy')
    nfr_cw = max(1, n_snapshots)
    cw_mm = np.lib.format.open_memmap(cw_path, mode='w+', dtype=np.float32, shape=(nfr_cw,) + E_c.shape)
    cw_frames = []
    for q in range(nfr_cw):
        tk = (q / nfr_cw) * (1.0 / (w_k[k_c] / 2 / np.pi))
        cw_mm[q] = np.real(E_c * np.exp(1j * w_k[k_c] * tk)).astype(np.float32)
        cw_frames.append({'x_start': 0.0, 'x_end': L_um, 'y_start': y0_um, 'y_end': y1_um, 'slide_i': 0,
                          'step': q, 'time': tk})
    cw_mm.flush()
    del cw_mm
    res = dict(r_c)
    res.update(scenario=label, method='stitch-pulse', frames=frames, frames_memmap=mm_path, cw_frames=cw_frames,
               cw_frames_memmap=cw_path, view_primary='transient', cw_only=False, Iavg=None, source_type='pulse',
               lambda_nm=lambda_nm, total_time=time.time() - t_total,
               spectrum=dict(lam_nm=lam_k, T=np.array(spec_T), P_out=np.array(spec_P),
                             weight=np.abs(S_k) / np.abs(S_k).max()),
               pulse=dict(cycles=pulse_cycles, s_fs=s_p * 1e15, tmax_fs=t_max * 1e15, nfreq=len(w_k),
                          dispersion=bool(pulse_dispersion)))
    if stack is not None:              # the stack at lambda0
        st = [dict(Ly) for Ly in stack]
        res['stack'], res['stack_custom'] = st, True
        res['layers'] = tuple([st[q]['t_um'] * 1e-6 if q < len(st) else 0.0 for q in range(3)] +
                              [complex(st[1]['n']).real if len(st) > 1 else
                               (complex(st[0]['n']).real if st else 1.333)])
    wgt = np.abs(S_k) ** 2
    res['transmission'] = float(np.sum(wgt * np.array(spec_T)) / np.sum(wgt))   # spectrally weighted
    return res


def run_beads_sliding(wg_mat, bead_mat, bead_d_um, dx_nm, save_frames, n_snapshots,
                      wg_thickness_um, lambda_nm, vcsel_waist, vcsel_tilt,
                      vcsel_offset, source_type, window_w_um, slide_um, place_bead=True,
                      t_aqueous_um=None, t_mucin_um=None, t_lipid_um=0.0, input_gap_um=0.0,
                      length_um=None, bead_x_um=None, bead_y_um=None, wg_n=None, bead_n=None,
                      n_aqueous=None, n_mucin=None, n_cornea=None, n_lipid=None,
                      polarization='s', curved=False, boundary='cpml', pulse_cycles=30.0,
                      cad=None, stack=None):
    """2D co-moving window (fdtd2d_core.py:930-1194): a window of window_w_um
    follows the wave down the guide in slides of slide_um.  Each slide rebuilds
    the window's materials at its x position, moves the fields and the psi of
    the CPML (all four edges) back by the slide (the last rows zero) and runs
    the slide's steps on the engine; the VCSEL (CW or Gaussian pulse) drives
    the first slide only.  The detector boxes and the time-domain Poynting
    planes count while their x lies in the window, so transmission is a ratio
    of pulse energies.  The reference keeps psi over the whole window, and the
    rolled psi keeps its value outside the absorber (b = 1, c = 0 there): the
    engine's window grid does the same (psi over every row along x).
    Supported: boundary='cpml', no CAD, flat geometry."""
    if str(boundary or 'cpml').lower() != 'cpml' or cad is not None or curved:
        raise NotImplementedError(f'lens_sensor_b200.run_beads_sliding: boundary={boundary!r} '
                                  f'cad={cad is not None} curved={curved}: only the CPML co-moving window '
                                  f'runs on the B200 engine')
    pol = 'p' if str(polarization).lower() in ('p', 'tm') else 's'
    t_total = time.time()
    t_aq_um = t_aqueous_um if t_aqueous_um is not None else T_AQ * 1e6
    wg_n = wg_n if wg_n is not None else n_at(wg_mat, lambda_nm)
    bead_n = bead_n if bead_n is not None else n_at(bead_mat, lambda_nm)
    n_aq_l = n_aqueous if n_aqueous is not None else n_at('aqueous', lambda_nm)
    n_mu_l = n_mucin if n_mucin is not None else n_at('mucin', lambda_nm)
    n_co_l = n_cornea if n_cornea is not None else cornea_default(lambda_nm)
    n_lip_l = n_lipid if n_lipid is not None else n_at('lipid', lambda_nm)
    L = (length_um * 1e-6) if length_um is not None else L_DEMO
    L_um = L * 1e6
    T_WG = wg_thickness_um * 1e-6
    LAM = lambda_nm * 1e-9
    label = f'WG-{wg_mat}_Bead-{bead_mat}_d{bead_d_um:g}_L{lambda_nm:g}' + ('' if place_bead else '_ref')
    dx = dx_nm * 1e-9
    dt = 0.5 * dx / (C0 * np.sqrt(2))
    NPML = 10
    src_ix = NPML + 2
    vd = float(input_gap_um or 0.0)
    air = air_path_um(vd, dx * 1e6)
    x_facet_um = src_ix * dx * 1e6 + air
    tear_m = TEAR_BUFFER
    y0_m = -tear_m
    H_total = T_WG + AIR_BUFFER + tear_m
    Nx, Ny = int(round(window_w_um * 1e-6 / dx)), int(round(H_total / dx))
    bx_um = bead_x_um if bead_x_um is not None else L_um / 2.0
    n_slides = int(np.ceil(L_um / slide_um))
    N_shift = int(round(slide_um * 1e-6 / dx))
    st, lossy, k = _stack_2d(wg_n, wg_thickness_um, t_lipid_um, n_lip_l, t_aq_um, n_aq_l, t_mucin_um, n_mu_l,
                             n_co_l, stack)
    bead = None
    if place_bead and bead_d_um:
        bead = Bead2D(bx_um, bead_d_um, complex(bead_n, k.get('bead', 0.0)) if lossy else bead_n, bead_y_um)
    f0 = C0 / LAM
    omega = 2 * np.pi * f0
    if source_type == 'pulse':       # exp(-((t - 3 s)/s)^2), s = pulse_cycles / f0 (fdtd2d_core.py:1107-1109)
        s_p = pulse_cycles / f0
        env = lambda t: np.exp(-(((t - 3 * s_p) / s_p) ** 2))
    else:
        env = E.cw_envelope(f0)
    iy_lo, iy_hi = int(round(tear_m / dx)), int(round((T_WG + tear_m) / dx))
    # detectors in global x (um); the input plane kept downstream of the source (flux.py:64-74)
    xi_g = _guard_in_plane(int(round(0.1 * L_um / (dx * 1e6))), max(src_ix, int(round(x_facet_um / (dx * 1e6)))),
                           int(round(L / dx))) * dx * 1e6
    det = ((xi_g, 'in'), (0.9 * L_um, 'out'))
    hw = max(1, int(round(min(DET_LEN / 2, 0.05 * L_um * 1e-6) / dx)))
    frames, mm_path, ez_mm, k_fr = [], None, None, 0
    safe = ''.join(c if (c.isalnum() or c in '-_.') else '_' for c in label)
    if save_frames:
        os.makedirs('results', exist_ok=True)
        mm_path = os.path.join('results', f'_stream_beads_{safe}_sliding.npy')
        ez_mm = np.lib.format.open_memmap(mm_path, mode='w+', dtype=np.float32,
                                          shape=(max(1, n_snapshots + n_slides + 4), Nx, Ny))
    sums = dict(in_P=0.0, out_P=0.0, **{q: 0.0 for q in ('in', 'out', 'src_up', 'src_dn')})
    grid = None
    t_start = time.time()
    for slide_i in range(n_slides):
        x_start_um = slide_i * slide_um
        if x_start_um >= L_um:
            break
        x_end_um = x_start_um + window_w_um
        src_active = slide_i == 0
        sp = Spec2D(pol, Nx, Ny, dx, st, tear_m, bead, npml=NPML, lam_nm=lambda_nm, waist_um=vcsel_waist,
                    length_m=L, vcsel_distance_um=vd, vcsel_offset_um=vcsel_offset, vcsel_tilt_deg=vcsel_tilt,
                    src_core_only=SRC_CORE_ONLY, x_start_um=x_start_um)
        geo = build_2d(sp)
        coef = {q: geo[q] for q in ('ce_e', 'ce_h', 'ca_x', 'ca_y', 'da_x', 'da_y') if q in geo}
        new = E.Grid2D(pol, Nx, Ny, dx, dt, coef, geo['cx'], geo['cy'], geo['src'] if src_active else None,
                       full_x=True)
        if grid is not None:         # fields and psi move with the window (fdtd2d_core.py:1093-1102)
            new.take_shifted(grid, N_shift if 0 < N_shift < Nx else 0)
        grid = new
        steps_slide = (int(window_w_um * 1e-6 * wg_n / C0 / dt) if src_active
                       else int(slide_um * 1e-6 * wg_n / C0 / dt)) + 200
        snap_every = max(1, steps_slide // max(1, n_snapshots // n_slides + 1))
        boxes, names, sxp = [], [], {}
        for xg, which in det:
            if x_start_um <= xg <= x_end_um:
                cl = int(round((xg - x_start_um) * 1e-6 / dx))
                boxes.append((max(0, cl - hw), min(Nx, cl + hw), iy_lo, iy_hi))
                names.append(which)
                if 1 <= cl < Nx - 1:
                    sxp[which] = cl
        if src_active:               # energy around the VCSEL pair (vcsel.py:158-166)
            sxp.update(src_up=src_ix - 1, src_dn=src_ix + 3)
        ep = E.Epi2D(grid, boxes=boxes, sx_planes=sxp, box_split=True)
        tab = E.StepTable(0, steps_slide, dt, geo['src']['omega'], omega, env)
        n = 0
        while n < steps_slide:
            nxt = min(steps_slide, (n // snap_every + 1) * snap_every)
            grid.step(tab, n, nxt - n, ep)
            n = nxt
            if save_frames and n % snap_every == 0 and k_fr < ez_mm.shape[0]:
                ez_mm[k_fr] = _field_2d(grid)
                frames.append({'x_start': x_start_um, 'x_end': x_end_um, 'y_start': y0_m * 1e6,
                               'y_end': (y0_m + H_total) * 1e6, 'slide_i': slide_i, 'step': n,
                               'time': time.time() - t_start})
                k_fr += 1
        box = ep.box_acc.double().cpu().numpy()
        for q, which in enumerate(names):
            sums[which + '_P'] += float(box[q])
        for which in sxp:
            sums[which] += ep.sx(which)
        del ep
    if ez_mm is not None:
        ez_mm.flush()
        del ez_mm
    total_time = time.time() - t_total
    P_in, P_out = sums['in_P'] * dx * dx, sums['out_P'] * dx * dx
    Tr_I = P_out / max(P_in, 1e-30)
    S_in, S_out, S_up, S_dn = sums['in'], sums['out'], sums['src_up'], sums['src_dn']
    Tr = S_out / S_in if abs(S_in) > 0 else Tr_I
    tr_def = 'poynting' if abs(S_in) > 0 else 'intensity'
    res = _result_dict(label, P_in, P_out, Tr, frames, total_time, bead_d_um, wg_mat, bead_mat, wg_n, bead_n,
                       wg_thickness_um, lambda_nm, vcsel_waist, vcsel_tilt, vcsel_offset, source_type, 'sliding',
                       place_bead, n_aq_l, n_mu_l, n_co_l, mm_path, t_aq_um, t_mucin_um, t_lipid_um, bx_um,
                       x_facet_um, L_um, pol, stack, n_lip_l)
    res['transmission_intensity'] = Tr_I
    res['transmission_def'] = tr_def
    # VCSEL pulse energies [J/m]: coupling only, no power scaling (fdtd2d_core.py:415-435, 1187-1188)
    p_emit, p_refl = (S_dn - S_up) * dx, -S_up * dx
    res.update(laser_power_mw=LASER_POWER_MW, vcsel_distance_um=vd, vcsel_air_um=float(air),
               vcsel_waist_um=float(vcsel_waist), x_facet_um=float(x_facet_um), p_src_si=None)
    if p_emit and p_emit > 0:
        res['coupling_efficiency'] = (S_in * dx) / p_emit
        res['facet_reflection'] = p_refl / p_emit
    return res


class FluxSum2D:
    """Plane DFTs summed over the windows that carry the plane (one running
    PlaneFluxDFT across windows, fdtd2d_core.py:1395, 1466-1469)."""

    def __init__(self, engine):
        self.E = engine
        self.acc, self.n = {}, {}

    def add(self, key, pairs, n):
        if key not in self.acc:
            self.acc[key] = [[sg, aE.clone(), aH.clone()] for sg, aE, aH in pairs]
            self.n[key] = 0
        else:
            for a, (sg, aE, aH) in zip(self.acc[key], pairs):
                a[1] += aE
                a[2] += aH
        self.n[key] += int(n)

    def has(self, key):
        return self.n.get(key, 0) > 0

    def flux(self, key):
        if not self.has(key):
            return float('nan')
        return self.E.plane_flux(self.acc[key], self.n[key])


def _field_2d(g):
    """Ez (TE) or Ey averaged onto the nodes (TM), fdtd2d_core.py:458-465."""
    if g.pol == 's':
        return g.view('ez').cpu().numpy()
    ey = g.view('ey').cpu().numpy()
    out = np.zeros((ey.shape[0], ey.shape[1] + 1), np.float32)
    out[:, 1:-1] = 0.5 * (ey[:, :-1] + ey[:, 1:])
    out[:, 0], out[:, -1] = ey[:, 0], ey[:, -1]
    return out


def _result_dict(label, P_in, P_out, Tr, frames, total_time, bead_d_um, wg_mat, bead_mat, wg_n, bead_n,
                 wg_th, lam, waist, tilt, off, src, method, place_bead, n_aq, n_mucin, n_cornea,
                 frames_memmap, t_aq_um, t_mu_um, t_lip_um, bead_x_um, x_wg_start_um, x_wg_end_um,
                 polarization, stack, n_lip):
    """Result keys of fdtd2d_core._result_dict (fdtd2d_core.py:2020-2049)."""
    t_aq = (t_aq_um * 1e-6) if t_aq_um is not None else T_AQ
    t_mu = (t_mu_um * 1e-6) if t_mu_um is not None else T_MU
    t_lip = (t_lip_um or 0.0) * 1e-6
    if stack is None:
        kp = dict(KAPPA or {})
        stack_out = []
        for nm, t, n, mat in (('Lipid', t_lip, n_lip, 'lipid'), ('Aqueous', t_aq, n_aq, 'aqueous'),
                              ('Mucin', t_mu, n_mucin, 'mucin')):
            if t * 1e6 > 1e-9:
                nc = complex(float(n), kp.get({'lipid': 'lip', 'aqueous': 'aq', 'mucin': 'mu'}[mat], 0.0))
                stack_out.append(dict(name=nm, t_um=t * 1e6, n=nc, kappa=nc.imag, mat=mat))
        layers = (t_lip, t_aq, t_mu, n_aq)
    else:
        stack_out = [dict(Ly) for Ly in stack]
        st = list(stack)
        layers = tuple([st[q]['t_um'] * 1e-6 if q < len(st) else 0.0 for q in range(3)] +
                       [complex(st[1]['n']).real if len(st) > 1 else (complex(st[0]['n']).real if st else 1.333)])
    return dict(scenario=label, P_in=P_in, P_out=P_out, transmission=Tr, frames=frames,
                frames_memmap=frames_memmap, stack=stack_out, stack_custom=stack is not None,
                total_time=total_time, layers=layers, n_aq=n_aq, n_mucin=n_mucin, n_cornea=n_cornea,
                wg_material=wg_mat, bead_material=bead_mat, wg_n=wg_n, bead_n=bead_n,
                bead_diameter_um=(bead_d_um if place_bead else 0.0), bead_x_um=bead_x_um,
                x_wg_start_um=x_wg_start_um, x_wg_end_um=x_wg_end_um, wg_thickness_um=wg_th,
                lambda_nm=lam, vcsel_waist=waist, vcsel_tilt=tilt, vcsel_offset=off, source_type=src,
                method=method, polarization=polarization)


def save_results(result, out_dir='results'):
    """PKL summary + beads_<scenario>_<method>_frames.npz with the keys the
    analyzer reads (fdtd2d_core.py:2085-2265)."""
    os.makedirs(out_dir, exist_ok=True)
    tag = f"{result['scenario']}_{result.get('method', 'full')}"
    summary = {q: v for q, v in result.items() if q not in ('frames', 'cad_region', 'Iavg', 'Ex_cw_amp', 'Ecw')}
    with open(f'{out_dir}/beads_{tag}.pkl', 'wb') as f:
        pickle.dump(summary, f)
    frames = result.get('frames')
    if not frames:
        return None
    n_fr = len(frames)
    ez = np.array(np.load(result['frames_memmap'], mmap_mode='r')[:n_fr])
    sx = next((s for s in (1, 2, 3, 4, 6, 8, 12, 16, 32) if ez.shape[1] // s <= 5000), 32)
    sy = next((s for s in (1, 2, 4, 8) if ez.shape[2] // s <= 2000), 8)
    meta = np.array([(fr['x_start'], fr['x_end'], fr['y_start'], fr['y_end'], fr['slide_i'], fr['time'],
                      fr.get('step', 0)) for fr in frames], dtype=np.float64)
    kw = dict(Ez=np.ascontiguousarray(ez[:, ::sx, ::sy]), meta=meta, scenario=result['scenario'],
              layers=np.array([np.real(v) for v in result['layers']], dtype=np.float64),
              bead_n=np.array([float(np.real(result.get('bead_n', 0.0)))]),
              bead_material=np.array([str(result.get('bead_material', ''))]),
              bead_x_um=np.array([result.get('bead_x_um', 0.0)]),
              bead_diameter_um=np.array([result.get('bead_diameter_um', 0.0)]),
              t_wg_um=np.array([result.get('wg_thickness_um', 5.0)]),
              x_wg_start_um=np.array([result.get('x_wg_start_um', 0.0) or 0.0]),
              x_wg_end_um=np.array([result.get('x_wg_end_um', 0.0) or 0.0]),
              polarization=np.array([str(result.get('polarization', 's'))]),
              lam_nm=np.array([result.get('lambda_nm', 850.0)]))
    # material table [core, layers, substrate] (fdtd2d_core.py:2055-2082)
    names5 = list(result.get('layer_names') or ['WG', 'Lipid', 'Aqueous', 'Mucin', 'Cornea'])
    st = list(result.get('stack') or [])
    if not result.get('stack_custom'):
        pos = {'lipid': 1, 'aqueous': 2, 'mucin': 3}
        st = [dict(Ly, name=str(names5[pos[Ly['mat']]])) if Ly.get('mat') in pos and len(names5) > 3
              else dict(Ly) for Ly in st]
        kw['material_names'] = np.array(names5)
        kw['material_indices'] = np.array([result['wg_n'], result.get('n_lip', N_LIPID), result['n_aq'],
                                           result['n_mucin'], result['n_cornea']], dtype=np.float64)
    else:
        kw['material_names'] = np.array([str(names5[0])] + [str(Ly['name']) for Ly in st] + [str(names5[-1])])
        kw['material_indices'] = np.array([float(np.real(result['wg_n']))] + [complex(Ly['n']).real for Ly in st]
                                          + [float(result['n_cornea'])], dtype=np.float64)
    kw.update(stack_names=np.array([L['name'] for L in st] or [''], dtype=str)[:len(st)],
              stack_t_um=np.array([L['t_um'] for L in st], dtype=np.float64),
              stack_n_re=np.array([complex(L['n']).real for L in st], dtype=np.float64),
              stack_n_im=np.array([complex(L['n']).imag for L in st], dtype=np.float64))
    cw_frames = result.get('cw_frames') or []
    cw_path = result.get('cw_frames_memmap')
    if cw_path and os.path.exists(cw_path) and cw_frames:
        kw['Ez_cw'] = np.array(np.load(cw_path, mmap_mode='r')[:len(cw_frames), ::sx, ::sy])
        kw['meta_cw'] = np.array([(fr['x_start'], fr['x_end'], fr['y_start'], fr['y_end'], fr['slide_i'],
                                   fr['time'], fr.get('step', 0)) for fr in cw_frames], dtype=np.float64)
    cw_only = bool(result.get('cw_only', False)) or result.get('method') == 'stitch'
    kw.update(has_transient=np.array([0 if cw_only else 1]),
              has_cw=np.array([1 if (cw_only or 'Ez_cw' in kw) else 0]),
              cw_only=np.array([1 if cw_only else 0]),
              view_primary=np.array([str(result.get('view_primary', 'transient'))]))
    if result.get('Iavg') is not None:
        kw['Iavg'] = np.asarray(result['Iavg'])[::sx, ::sy].astype(np.float32)
        kw['iavg_full'] = np.array([1])
    if result.get('Ex_cw_amp') is not None:
        kw['Ex_cw_amp'] = np.asarray(result['Ex_cw_amp'])[::sx, ::sy].astype(np.complex64)
    if result.get('p_in_si') is not None:
        kw['p_in_si'] = np.array([float(result['p_in_si'])])
        kw['p_in_unit'] = np.array([str(result.get('p_in_unit', 'W/m'))])
    for q in ('laser_power_mw', 'p_src_si', 'coupling_efficiency', 'facet_reflection', 'vcsel_distance_um',
              'vcsel_air_um', 'vcsel_waist_um', 'x_facet_um'):
        v = result.get(q)
        if v is not None and np.isfinite(float(v)):
            kw[q] = np.array([float(v)])
    spec = result.get('spectrum')
    if spec:                           # Fourier stitch: spectrum and pulse (fdtd2d_core.py:2229-2236)
        pu = result.get('pulse') or {}
        kw.update(spec_lam_nm=np.asarray(spec['lam_nm'], dtype=np.float64),
                  spec_T=np.asarray(spec['T'], dtype=np.float64),
                  spec_weight=np.asarray(spec['weight'], dtype=np.float64),
                  pulse_cycles=np.array([pu.get('cycles', 0.0)]), pulse_tmax_fs=np.array([pu.get('tmax_fs', 0.0)]),
                  pulse_dispersion=np.array([int(bool(pu.get('dispersion', True)))]))
    npz = f'{out_dir}/beads_{tag}_frames.npz'
    np.savez_compressed(npz, **kw)
    # the temporary frame stream files go once the NPZ is written (fdtd2d_core.py:2243-2265)
    for path in (cw_path, result.get('frames_memmap')):
        if path and os.path.exists(path):
            os.remove(path)
    return npz
