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
    """2D TE/TM full-domain CW solve (fdtd2d_core.py:531-927) on the GPU engine."""
    if method != 'full' or str(boundary).lower() != 'cpml' or source_type != 'cw' or cad is not None or curved:
        raise NotImplementedError(f'lens_sensor_b200.run_beads: method={method!r} boundary={boundary!r} '
                                  f'source_type={source_type!r} cad={cad is not None} curved={curved}: '
                                  f'only the full-domain CPML CW path runs on the B200 engine')
    global TEAR_BUFFER
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
    ez = np.load(result['frames_memmap'], mmap_mode='r')[:n_fr]
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
        kw['Ez_cw'] = np.ascontiguousarray(np.load(cw_path, mmap_mode='r')[:len(cw_frames), ::sx, ::sy])
        kw['meta_cw'] = np.array([(fr['x_start'], fr['x_end'], fr['y_start'], fr['y_end'], fr['slide_i'],
                                   fr['time'], fr.get('step', 0)) for fr in cw_frames], dtype=np.float64)
    kw.update(has_transient=np.array([1]), has_cw=np.array([1 if 'Ez_cw' in kw else 0]),
              cw_only=np.array([0]), view_primary=np.array([str(result.get('view_primary', 'transient'))]))
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
    npz = f'{out_dir}/beads_{tag}_frames.npz'
    np.savez_compressed(npz, **kw)
    return npz
