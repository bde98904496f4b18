"""Post-processing on the GPU: the reference's post_processor.py
(utility_scripts/post_processor.py) with its spectra computed by the
library's batched DFT kernel (aem_dft_batch).

The reference reads every series of the run's .dat files, zero-pads each by
`padding` times its length, takes numpy's FFT of all of them
(post_processor.py:160-215), forms S-parameters, radar cross sections or
realised gain (:217-266) and writes the bins inside the pulse's trusted band
to CSV files (:268-388).  Only the band's bins reach the CSVs, so here each
series' spectrum is evaluated at exactly those FFT bins, k / ((padding+1)
N dt) for k in the band: the same sums, in FP64, without the padding.  All
series of a run go through one batched launch.  The formulas, the band
selection, the CSV headers and the number format (numpy.savetxt) are the
reference's.

`post_process` takes the reference script's configuration variables as
arguments (same names, same meaning); `post_process_kmax` does the same for
the constant-k post-processor (utility_scripts/post_processor_kmax.py).  SPICE ports are outside this build:
decks with SPICE ports or spice_excitation are rejected.  There is no CPU
path: the spectra need the CUDA library and a GPU.
"""
import os

import numpy as np

IMPED_FREE = 376.730313  # post_processor.py:71


def _tok(line, c):
    return float(line.split()[c])


def read_dat(path):
    """The blocks of a standard-solver .dat that the post-processor reads,
    at its fixed line offsets (post_processor.py:45-159), as float64."""
    with open(path) as f:
        L = f.read().splitlines()
    d = dict(lines=L, time_step=_tok(L[4], 3), steps=int(_tok(L[5], 5)), pulse_freq=_tok(L[7], 3) / 1e9,
             pulse_type=_tok(L[8], 3), num_angles=int(_tok(L[13], 6)), num_ports=int(_tok(L[14], 5)),
             num_spice_ports=int(_tok(L[15], 5)), sim=[int(_tok(L[16], c)) for c in (2, 3, 4)],
             size=[int(_tok(L[q], 3)) for q in (0, 1, 2)], step=[_tok(L[3], c) for c in (3, 4, 5)])
    return d


def _block(L, start, n):
    return np.array([float(v) for v in L[start:start + n]], dtype=np.float64)


def _line_values(line):
    v = [float(t) for t in line.split()]
    return v[0] if len(v) == 1 else np.array(v)


def _angle_str(x):
    return str(np.float64(x))


def post_process(simulation_type="plane wave", data_filename="data.dat", clear_filename="clear.dat",
                 metal_filename="metal.dat", IGP_full_clear_filename="IGP_full_clear.dat", padding=10,
                 use_metal=False, use_IGP_full_clear=False, S_parameter_output_file_name="S_parameters.csv",
                 Scattering_output_file_name="Scattering_Far_Field.csv",
                 Antenna_gain_output_file_name="Realized_antenna_gain.csv", spice_excitation=False, directory=None,
                 device=None):
    """Run the reference post-processing of the .dat files in `directory`
    (default: the current directory) and write its CSV files there.
    Returns the paths written."""
    import torch

    import alpineem_b200 as ab

    if spice_excitation:
        raise NotImplementedError("SPICE excitation is outside this build")
    if simulation_type not in ("plane wave", "antenna"):
        raise ValueError("simulation_type must be 'plane wave' or 'antenna'")
    path = (lambda f: os.path.join(directory, f)) if directory else (lambda f: f)
    dev = torch.device(device) if device else torch.device("cuda", torch.cuda.current_device())
    plane = simulation_type == "plane wave"

    # ---- header values and blocks, post_processor.py:45-159
    D = read_dat(path(data_filename))
    L = D["lines"]
    time_step, N = D["time_step"], D["steps"]
    if D["pulse_type"] == 1:
        pulse_bounds = [0.0, 2.146]
    elif D["pulse_type"] == 2:
        pulse_bounds = [0.183, 3.087]
    else:
        raise ValueError("pulse type %g has no trusted band in the reference post-processor" % D["pulse_type"])
    num_angles, num_ports, num_spice = D["num_angles"], D["num_ports"], D["num_spice_ports"]
    if num_spice:
        raise NotImplementedError("SPICE ports are outside this build")
    sx, sy, sz = D["sim"]
    size_x, size_y, size_z = D["size"]
    step_x, step_y, step_z = D["step"]
    wave_port_num = 2
    area = None
    if sy + sz == 2:
        area = size_z * step_z * size_y * step_y
    if sx + sz == 2:
        area = size_z * step_z * size_x * step_x
    if sx + sy == 2:
        area = size_y * step_y * size_x * step_x
    if sx + sy + sz < 2:
        wave_port_num = 0
        area = 1
    port_number_int = None
    if not plane:
        wave_port_num = 0
        port_number_int = int(_tok(L[17], 5))

    C = read_dat(path(clear_filename))["lines"] if plane else None
    M = read_dat(path(metal_filename))["lines"] if (plane and use_metal) else None

    series = []          # rows of the batched DFT
    def add(x):
        series.append(x)
        return len(series) - 1

    inc_row = add(_block(L, 18, N))
    skip = 18 + N
    wave_rows = []
    for i in range(wave_port_num):
        skip += 1
        r0 = add(_block(L, skip, N))
        r1 = add(_block(C, skip, N)) if plane else None
        r2 = add(_block(M, skip, N)) if M is not None else None
        wave_rows.append((r0, r1, r2))
        skip += N
    ff_rows, ff_angles = [], []
    for i in range(2 * num_angles):
        skip += 1
        if i % 2 == 0:
            a = L[skip].split()
            ff_angles.append((float(a[0]), float(a[1])))
        skip += 1
        ff_rows.append((add(_block(L, skip, N)), add(_block(C, skip, N)) if plane else None))
        skip += N
    skip_clear = skip + 1
    tc_clear = []
    for i in range(num_angles):
        if plane:
            tc_clear.append(_line_values(C[skip_clear]))
            skip_clear += 1
    pc_row = None
    if num_angles > 0 and plane:
        src = read_dat(path(IGP_full_clear_filename))["lines"] if use_IGP_full_clear else C
        pc_row = add(_block(src, skip_clear + 1, N))
    imped, v_rows = [], []
    for i in range(num_ports + num_spice):
        skip += 1
        imped.append(_line_values(L[skip]))
        skip += 1
        v_rows.append(add(_block(L, skip, N)))
        skip += N
    skip += 1
    tc = []
    for i in range(num_angles):
        tc.append(_line_values(L[skip]))
        skip += 1

    # ---- trusted band and the spectra at its FFT bins (:160-215, :299-307)
    n_pad = int((padding + 1) * N)
    freq_all = np.fft.fftfreq(n_pad, time_step)
    low, high = pulse_bounds[0] * D["pulse_freq"] * 1e9, pulse_bounds[1] * D["pulse_freq"] * 1e9
    rec = np.nonzero((freq_all >= low) & (freq_all <= high))[0]
    lo, hi = int(rec.min()), int(rec.max())
    freq = freq_all[lo:hi + 1]
    x = torch.from_numpy(np.stack(series)).to(dev)
    fr = torch.from_numpy(freq.copy()).to(dev)
    spec = ab.dft_batch(x, time_step, fr).cpu().numpy()
    F = lambda r: spec[r] if r is not None else np.zeros(len(freq), dtype=complex)
    inc_f = F(inc_row)

    # ---- S-parameters and far-field quantities (:217-266)
    S, scatter = [], []
    if plane:
        for i, (r0, r1, r2) in enumerate(wave_rows):
            if i == 0:
                S.append(-1 * (F(r0) - F(r1)) / (F(r2) - F(r1)))
            else:
                S.append(-1 * (F(r0) - F(r2)) / (F(r1) - F(r2)))
        for i in range(num_ports + num_spice):
            port_pwave = F(v_rows[i]) / np.sqrt(np.real(imped[i]))
            if wave_port_num != 0:
                waveport_pwave = F(wave_rows[0][1]) * np.sqrt(area / np.real(IMPED_FREE))
            else:
                waveport_pwave = inc_f * np.sqrt(area / np.real(IMPED_FREE))
            S.append(port_pwave / waveport_pwave)
        for i in range(2 * num_angles):
            t = i // 2
            normal_phase = np.exp(1j * 2 * np.pi * freq * tc[t] - 1j * np.pi / 2)
            clear_phase = np.exp(1j * 2 * np.pi * freq * tc_clear[t] - 1j * np.pi / 2)
            scatter.append((F(ff_rows[i][0]) * normal_phase - F(ff_rows[i][1]) * clear_phase) / F(pc_row))
    else:
        for i in range(num_ports + num_spice):
            if i == port_number_int - 1:
                S.append((F(v_rows[i]) - inc_f) / inc_f)
            else:
                S.append((F(v_rows[i]) / np.sqrt(np.real(imped[i]))) /
                         (inc_f / np.sqrt(np.real(imped[port_number_int - 1]))))
        for i in range(2 * num_angles):
            scatter.append(F(ff_rows[i][0]))

    # ---- CSV files (:268-388)
    written = []
    if num_ports + num_spice + wave_port_num > 0:
        out = [freq / 1e9]
        for s in S:
            out.append(20 * np.log10(np.abs(s)))
            out.append(np.angle(s))
        head = ["Frequency (GHz)"]
        if wave_port_num > 0 and plane:
            head += ["Wave Refl (dB)", "Wave Refl (rad)", "Wave Trans (dB)", "Wave Trans (rad)"]
        for i in range(num_ports):
            if plane:
                if wave_port_num != 0:
                    name = "S_lumpedport%d:inc_waveport" % (i + 1)
                else:
                    name = ("A_e for port %d - Vport/Einc phase center info: Vport fdtd grid (centered) port "
                            "location & Einc location" % (i + 1))
            else:
                name = "S%d:%d" % (i + 1, port_number_int)
            head += ["%s (dB)" % name, "%s (rad)" % name]
        fn = path(S_parameter_output_file_name)
        np.savetxt(fn, np.transpose(out), delimiter=",", header=", ".join(head), comments="")
        written.append(fn)
    if num_angles > 0:
        out = [freq / 1e9]
        head = ["Frequency (GHz)"]
        if plane:
            for s in scatter:
                out.append(20 * np.log10(np.abs(s)) + 10 * np.log10(4 * np.pi))
                out.append(np.angle(s))
            for th, ph in ff_angles:
                t, p = _angle_str(th), _angle_str(ph)
                head += ["RCS Theta Pol: Theta=%s & Phi=%s (dBsm)" % (t, p),
                         "RCS Theta Pol: Theta=%s & Phi=%s (rad of rEfar/Einc - phase centered at ff origin)" % (t, p),
                         "RCS Phi Pol: Theta=%s & Phi=%s (dBsm)" % (t, p),
                         "RCS Phi Pol: Theta=%s & Phi=%s (rad of rEfar/Einc - phase centered at ff origin)" % (t, p)]
            fn = path(Scattering_output_file_name)
        else:
            p_ant = np.abs(inc_f) ** 2 / (2 * np.real(imped[port_number_int - 1]))
            for i, s in enumerate(scatter):
                out.append(10 * np.log10(4 * np.pi * np.abs(s) ** 2 / (2 * IMPED_FREE * p_ant)))
                normal_phase = np.exp(1j * 2 * np.pi * freq * tc[i // 2] - 1j * np.pi / 2)
                out.append(np.angle(s * normal_phase / inc_f))
            for th, ph in ff_angles:
                t, p = _angle_str(th), _angle_str(ph)
                head += ["G_r Theta Pol: Theta=%s & Phi=%s (dB)" % (t, p),
                         "G_r Theta Pol: Theta=%s & Phi=%s (rad of rEfar/Vinc - eEfar phase centered at ff origin & "
                         "Vinc phase centered on fdtd grid port location)" % (t, p),
                         "G_r Phi Pol: Theta=%s & Phi=%s (dB)" % (t, p),
                         "G_r Phi Pol: Theta=%s & Phi=%s (rad of rEfar/Vinc- eEfar phase centered at ff origin & "
                         "Vinc phase centered on fdtd grid port location)" % (t, p)]
            fn = path(Antenna_gain_output_file_name)
        np.savetxt(fn, np.transpose(out), delimiter=",", header=", ".join(head), comments="")
        written.append(fn)
    return written


def _cblock(L, start, n):
    a = np.array([[float(t) for t in ln.split()[:2]] for ln in L[start:start + n]], dtype=np.float64)
    return a[:, 0] + 1j * a[:, 1]


def post_process_kmax(simulation_type="plane wave", data_filename="data-k.dat", clear_filename="clear-k.dat",
                      metal_filename="metal-k.dat", padding=10, use_metal=False,
                      S_parameter_output_file_name="S_parameters_k.csv",
                      Scattering_output_file_name="Scattering_Far_Field_k.csv",
                      Antenna_gain_output_file_name="Realized_antenna_gain_k.csv", dB_rule=20, spice_excitation=False,
                      directory=None, device=None):
    """The constant-k post-processor (utility_scripts/post_processor_kmax.py)
    on the GPU: complex series (two columns), two TE and two TM wave ports,
    the band where the incident spectrum is within `dB_rule` dB of its peak
    (:300-306), TE/TM projections with the cosine of the propagation angle
    (:226-236).  The phase-centre incident of the far field is formed as the
    reference forms it (:300-366): the time series times coefficients indexed
    by the FFT frequency grid, then transformed.  Returns the paths written."""
    import torch

    import alpineem_b200 as ab

    if spice_excitation:
        raise NotImplementedError("SPICE excitation is outside this build")
    if simulation_type not in ("plane wave", "antenna"):
        raise ValueError("simulation_type must be 'plane wave' or 'antenna'")
    path = (lambda f: os.path.join(directory, f)) if directory else (lambda f: f)
    dev = torch.device(device) if device else torch.device("cuda", torch.cuda.current_device())
    plane = simulation_type == "plane wave"
    with open(path(data_filename)) as f:
        L = f.read().splitlines()
    time_step, N = _tok(L[4], 3), int(_tok(L[5], 5))
    num_angles, num_ports, num_spice = int(_tok(L[13], 6)), int(_tok(L[14], 5)), int(_tok(L[15], 5))
    if num_spice:
        raise NotImplementedError("SPICE ports are outside this build")
    wave_port_num = 4
    sx, sy, sz = (int(_tok(L[16], c)) for c in (2, 3, 4))
    k_direction = int(_tok(L[16], 5))
    size_x, size_y, size_z = (int(_tok(L[q], 3)) for q in (0, 1, 2))
    step_x, step_y, step_z = (_tok(L[3], c) for c in (3, 4, 5))
    area = None
    if sy + sz == 2:
        area = size_z * step_z * size_y * step_y
    if sx + sz == 2:
        area = size_z * step_z * size_x * step_x
    if sx + sy == 2:
        area = size_y * step_y * size_x * step_x
    k1, k2 = _tok(L[18], 0), _tok(L[18], 1)
    mode_type = _tok(L[19], 10)
    port_number_int = int(_tok(L[20], 5)) if not plane else None
    C = open(path(clear_filename)).read().splitlines() if plane else None
    M = open(path(metal_filename)).read().splitlines() if (plane and use_metal) else None

    inc = _cblock(L, 21, N)
    skip = 21 + N
    waves = []
    for i in range(wave_port_num):
        skip += 1
        waves.append((_cblock(L, skip, N), _cblock(C, skip, N) if plane else None,
                      _cblock(M, skip, N) if M is not None else None))
        skip += N
    ffs, ff_angles = [], []
    for i in range(2 * num_angles):
        skip += 1
        if i % 2 == 0:
            a = L[skip].split()
            ff_angles.append((float(a[0]), float(a[1])))
        skip += 1
        ffs.append((_cblock(L, skip, N), _cblock(C, skip, N) if plane else None))
        skip += N
    skip_clear = skip + 1
    tc_clear = []
    for i in range(num_angles):
        if plane:
            tc_clear.append(_line_values(C[skip_clear]))
            skip_clear += 1
    Exyz = None
    if num_angles > 0 and plane:
        Exyz = []
        for c in range(3):
            Exyz.append(_cblock(C, skip_clear + 1, N))
            skip_clear += N
    imped, volts = [], []
    for i in range(num_ports + num_spice):
        skip += 1
        imped.append(_line_values(L[skip]))
        skip += 1
        volts.append(_cblock(L, skip, N))
        skip += N
    skip += 1
    tc = []
    for i in range(num_angles):
        tc.append(_line_values(L[skip]))
        skip += 1

    def spectra(rows, freqs):
        x = torch.from_numpy(np.stack([v for r in rows for v in (r.real, r.imag)])).to(dev)
        z = ab.dft_batch(x, time_step, torch.from_numpy(np.ascontiguousarray(freqs)).to(dev)).cpu().numpy()
        return [z[2 * q] + 1j * z[2 * q + 1] for q in range(len(rows))]

    # band: bins within dB_rule of the incident spectrum's peak (:300-306)
    n_pad = int((padding + 1) * N)
    freq_all = np.fft.fftfreq(n_pad, time_step)
    inc_all = spectra([inc], freq_all)[0]
    max_amp = np.max(np.abs(inc_all))
    db_down_boundary = max_amp / 10 ** (dB_rule / 10)
    index = np.where((np.abs(inc_all) >= db_down_boundary) & (freq_all >= 0.0))
    lo, hi = int(np.min(index)), int(np.max(index))
    freq = freq_all[lo:hi + 1]
    inc_f = inc_all[lo:hi + 1]

    rows, slot = [], {}
    def want(key, r):
        if r is not None:
            slot[key] = len(rows)
            rows.append(r)
    for i, (d, c, m) in enumerate(waves):
        want(("w", 0, i), d)
        want(("w", 1, i), c)
        want(("w", 2, i), m)
    for i, (d, c) in enumerate(ffs):
        want(("f", 0, i), d)
        want(("f", 1, i), c)
    for i, v in enumerate(volts):
        want(("v", i), v)
    spec = spectra(rows, freq) if rows else []
    zero = np.zeros(len(freq), dtype=complex)
    W = lambda j, i: spec[slot[("w", j, i)]] if ("w", j, i) in slot else zero
    FF = lambda j, i: spec[slot[("f", j, i)]]
    V = lambda i: spec[slot[("v", i)]]

    k = 2 * np.pi * freq / 299792458
    cos_ang = np.ones_like(k, dtype=float)
    if k1 != 0 or k2 != 0:
        arg = np.maximum(k ** 2 - k1 ** 2 - k2 ** 2, 0)
        with np.errstate(divide="ignore", invalid="ignore"):
            cos_ang = np.where(k != 0, np.sqrt(arg) / k, 1)
    cos_ang = np.clip(cos_ang, 1e-12, 1.0)

    S, scatter = [], []
    if plane:
        if mode_type == 0:
            S.append(-1 * (W(0, 0) - W(1, 0)) / (W(2, 0) - W(1, 0)))
            S.append(-1 * (W(0, 1) - W(1, 1)) / (W(2, 0) - W(1, 0)) / cos_ang)
            S.append(-1 * (W(0, 2) - W(2, 2)) / (W(1, 2) - W(2, 2)))
            S.append(-1 * (W(0, 3) - W(2, 3)) / (W(1, 2) - W(2, 2)) / cos_ang)
            inc_place_holder = W(1, 0)
        elif mode_type == 1:
            S.append(-1 * (W(0, 0) - W(1, 0)) / (W(2, 1) - W(1, 1)) * cos_ang)
            S.append(-1 * (W(0, 1) - W(1, 1)) / (W(2, 1) - W(1, 1)))
            S.append(-1 * (W(0, 2) - W(2, 2)) / (W(1, 3) - W(2, 3)) * cos_ang)
            S.append(-1 * (W(0, 3) - W(2, 3)) / (W(1, 3) - W(2, 3)))
            inc_place_holder = W(1, 1)
        else:
            raise ValueError("mode type %g is neither TE (0) nor TM (1)" % mode_type)
        for i in range(num_ports + num_spice):
            port_pwave = V(i) / np.sqrt(np.real(imped[i]))
            if mode_type == 0:
                waveport_pwave = inc_place_holder * np.sqrt(area / np.real(IMPED_FREE))
            else:
                waveport_pwave = inc_place_holder * np.sqrt(area / (np.real(IMPED_FREE) * cos_ang ** 2))
            S.append(port_pwave / waveport_pwave)
        if num_angles > 0:
            # projection coefficients (:312-366) on the full FFT grid
            import numpy.lib.scimath as scimath
            kf = 2 * np.pi * freq_all / 299792458
            k3 = scimath.sqrt(kf ** 2 - k1 ** 2 - k2 ** 2)
            k12 = np.sqrt(k1 ** 2 + k2 ** 2)
            kf = np.where(kf == 0, 1e-6, kf)
            sgn = 2 * k_direction - 1
            normal = k1 == 0 and k2 == 0
            with np.errstate(divide="ignore", invalid="ignore"):
                if sy + sz == 2:
                    if mode_type == 0:
                        cx, cy, cz = (0, sgn, 0) if normal else (0, k2 / k12 * sgn, -k1 / k12 * sgn)
                    else:
                        cx, cy, cz = (0, 0, sgn) if normal else (k12 / kf * sgn * -1.0, k3 * k1 / (kf * k12),
                                                                 k3 * k2 / (kf * k12))
                if sx + sz == 2:
                    if mode_type == 0:
                        cx, cy, cz = (sgn * -1, 0, 0) if normal else (-k2 / k12 * sgn, 0, k1 / k12 * sgn)
                    else:
                        cx, cy, cz = (0, 0, sgn) if normal else (k3 * k1 / (kf * k12), k12 / kf * sgn * -1.0,
                                                                 k3 * k2 / (kf * k12))
                if sx + sy == 2:
                    if mode_type == 0:
                        cx, cy, cz = (0, sgn * -1, 0) if normal else (k2 / k12 * sgn, -k1 / k12 * sgn, 0)
                    else:
                        cx, cy, cz = (sgn, 0, 0) if normal else (k3 * k1 / (kf * k12), k3 * k2 / (kf * k12),
                                                                 k12 / kf * sgn * -1.0)
            pad = np.zeros(n_pad - N, dtype=complex)
            Ep = [np.concatenate((e, pad)) for e in Exyz]
            pc_time = (Ep[0] * cx + Ep[1] * cy + Ep[2] * cz)[:N]
            pc_f = spectra([np.asarray(pc_time, dtype=complex)], freq)[0]
            for i in range(2 * num_angles):
                t = i // 2
                normal_phase = np.exp(1j * 2 * np.pi * freq * tc[t] - 1j * np.pi / 2)
                clear_phase = np.exp(1j * 2 * np.pi * freq * tc_clear[t] - 1j * np.pi / 2)
                scatter.append((FF(0, i) * normal_phase - FF(1, i) * clear_phase) / pc_f)
    else:
        for i in range(wave_port_num):
            port_pwave = inc_f / np.sqrt(np.real(imped[port_number_int - 1]))
            if i in (0, 2):
                waveport_pwave = W(0, i) * np.sqrt(area / np.real(IMPED_FREE))
            else:
                waveport_pwave = W(0, i) * np.sqrt(area / (np.real(IMPED_FREE) * cos_ang ** 2))
            S.append(waveport_pwave / port_pwave)
        for i in range(num_ports + num_spice):
            if i == port_number_int - 1:
                S.append((V(i) - inc_f) / inc_f)
            else:
                S.append((V(i) / np.sqrt(np.real(imped[i]))) /
                         (inc_f / np.sqrt(np.real(imped[port_number_int - 1]))))
        for i in range(2 * num_angles):
            scatter.append(FF(0, i))

    written = []
    out = [freq / 1e9]
    for sv in S:
        out.append(20 * np.log10(np.abs(sv)))
        out.append(np.angle(sv))
    head = ["Frequency (GHz)"]
    if plane:
        head += ["Wave Refl TE (dB)", "Wave Refl TE (rad)", "Wave Refl TM (dB)", "Wave Refl TM (rad)",
                 "Wave Trans TE (dB)", "Wave Trans TE (rad)", "Wave Trans TM (dB)", "Wave Trans TM (rad)"]
    else:
        for w in ("S_TEwaveport1", "S_TMwaveport1", "S_TEwaveport2", "S_TMwaveport2"):
            head += ["%s:lumpedport%d (dB)" % (w, port_number_int), "%s:lumpedport%d (rad)" % (w, port_number_int)]
    for i in range(num_ports):
        name = "S_lumpedport%d:inc_waveport" % (i + 1) if plane else "S%d:%d" % (i + 1, port_number_int)
        head += ["%s (dB)" % name, "%s (rad)" % name]
    fn = path(S_parameter_output_file_name)
    np.savetxt(fn, np.transpose(out), delimiter=",", header=", ".join(head), comments="")
    written.append(fn)
    if num_angles > 0:
        out = [freq / 1e9]
        head = ["Frequency (GHz)"]
        if plane:
            for sv in scatter:
                out.append(20 * np.log10(np.abs(sv)) + 10 * np.log10(4 * np.pi))
                out.append(np.angle(sv))
            for th, ph in ff_angles:
                t, p = _angle_str(th), _angle_str(ph)
                head += ["RCS Theta Pol: Theta=%s & Phi=%s (dBsm)" % (t, p),
                         "RCS Theta Pol: Theta=%s & Phi=%s (rad of rEfar/Einc - phase centered at ff origin)" % (t, p),
                         "RCS Phi Pol: Theta=%s & Phi=%s (dBsm)" % (t, p),
                         "RCS Phi Pol: Theta=%s & Phi=%s (rad of rEfar/Einc - phase centered at ff origin)" % (t, p)]
            fn = path(Scattering_output_file_name)
        else:
            p_ant = np.abs(inc_f) ** 2 / (2 * np.real(imped[port_number_int - 1]))
            for i, sv in enumerate(scatter):
                out.append(10 * np.log10(4 * np.pi * np.abs(sv) ** 2 / (2 * IMPED_FREE * p_ant)))
                normal_phase = np.exp(1j * 2 * np.pi * freq * tc[i // 2] - 1j * np.pi / 2)
                out.append(np.angle(sv * normal_phase / inc_f))
            for th, ph in ff_angles:
                t, p = _angle_str(th), _angle_str(ph)
                head += ["G_r Theta Pol: Theta=%s & Phi=%s (dB)" % (t, p),
                         "G_r Theta Pol: Theta=%s & Phi=%s (rad of rEfar/Vinc - eEfar phase centered at ff origin & "
                         "Vinc phase centered on fdtd grid port location)" % (t, p),
                         "G_r Phi Pol: Theta=%s & Phi=%s (dB)" % (t, p),
                         "G_r Phi Pol: Theta=%s & Phi=%s (rad of rEfar/Vinc- eEfar phase centered at ff origin & "
                         "Vinc phase centered on fdtd grid port location)" % (t, p)]
            fn = path(Antenna_gain_output_file_name)
        np.savetxt(fn, np.transpose(out), delimiter=",", header=", ".join(head), comments="")
        written.append(fn)
    return written


def main(argv=None):
    """Command line: python -m alpineem_b200.postprocess [--antenna] [--padding P]
    [--metal] [--igp-full-clear] [--dir D] -- the reference script's
    settings as flags; file names are the reference's defaults."""
    import argparse
    ap = argparse.ArgumentParser(description="GPU post-processing of AlpineEM .dat files")
    ap.add_argument("--antenna", action="store_true", help="simulation_type='antenna' (default 'plane wave')")
    ap.add_argument("--padding", type=int, default=10)
    ap.add_argument("--metal", action="store_true", help="use_metal=True")
    ap.add_argument("--igp-full-clear", action="store_true", help="use_IGP_full_clear=True")
    ap.add_argument("--dir", default=None)
    ap.add_argument("--kmax", action="store_true", help="the constant-k post-processor (data-k.dat, ...)")
    ap.add_argument("--db-rule", type=int, default=20, help="kmax: band within this many dB of the incident peak")
    a = ap.parse_args(argv)
    st = "antenna" if a.antenna else "plane wave"
    if a.kmax:
        files = post_process_kmax(st, padding=a.padding, use_metal=a.metal, dB_rule=a.db_rule, directory=a.dir)
    else:
        files = post_process(st, padding=a.padding, use_metal=a.metal, use_IGP_full_clear=a.igp_full_clear,
                             directory=a.dir)
    for fn in files:
        print(fn)


if __name__ == "__main__":
    main()
