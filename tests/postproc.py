"""Restatement of the reference post-processor's arithmetic
(utility_scripts/post_processor.py), used to turn .dat files into the
example CSV columns without importing the reference.  Line offsets and
formulas follow the cited lines; the reference file itself is run unchanged
by tests/test_oracle_golden.py where the reference checkout exists.
"""
import numpy as np


def _lines(path):
    with open(path) as f:
        return f.read().splitlines()


def _col(line, c):
    return float(line.split()[c])


def parse_dat(path):
    """Blocks of a standard-solver .dat by the post-processor's fixed line
    offsets (post_processor.py:45-159)."""
    L = _lines(path)
    out = dict(time_step=_col(L[4], 3), steps=int(_col(L[5], 5)), pulse_freq=_col(L[7], 3) / 1e9,
               pulse_type=int(_col(L[8], 3)), num_angles=int(_col(L[13], 6)), num_ports=int(_col(L[14], 5)),
               sim=[int(_col(L[16], c)) for c in (2, 3, 4)], size=[int(_col(L[q], 3)) for q in (0, 1, 2)],
               step=[_col(L[3], c) for c in (3, 4, 5)])
    T = out["steps"]
    pos = 18
    out["inc"] = np.array([float(x) for x in L[pos:pos + T]])
    pos += T
    nwave = 2 if sum(out["sim"]) == 2 else 0
    waves = []
    for _ in range(nwave):
        pos += 1
        waves.append(np.array([float(x) for x in L[pos:pos + T]]))
        pos += T
    out["waves"] = waves
    ff, ang = [], []
    for q in range(2 * out["num_angles"]):
        pos += 1
        a = L[pos].split()
        if q % 2 == 0:
            ang.append((float(a[0]), float(a[1])))
        pos += 1
        ff.append(np.array([float(x) for x in L[pos:pos + T]]))
        pos += T
    out["ff"], out["angles"] = ff, ang
    ports, imp = [], []
    for _ in range(out["num_ports"]):
        pos += 1
        imp.append(float(L[pos]))
        pos += 1
        ports.append(np.array([float(x) for x in L[pos:pos + T]]))
        pos += T
    out["ports"], out["imped"] = ports, imp
    tc = []
    if out["num_angles"] > 0:
        pos += 1
        for _ in range(out["num_angles"]):
            tc.append(float(L[pos]))
            pos += 1
    out["time_corr"] = tc
    if out["num_angles"] > 0 and pos < len(L) and L[pos].strip().startswith("incident for far field"):
        pos += 1
        out["inc_ff_pc"] = np.array([float(x) for x in L[pos:pos + T]])
    return out


def _band(d, n):
    freq = np.fft.fftfreq(n, d["time_step"])
    bounds = [0.0, 2.146] if d["pulse_type"] == 1 else [0.183, 3.087]  # post_processor.py:52-55
    lo, hi = bounds[0] * d["pulse_freq"] * 1e9, bounds[1] * d["pulse_freq"] * 1e9
    idx = np.nonzero((freq >= lo) & (freq <= hi))[0]
    return freq, idx.min(), idx.max()


def _fft(x, padding):
    return np.fft.fft(np.concatenate((x, np.zeros(len(x) * padding))))  # post_processor.py:163-215


def plane_wave_sparams(data, clear, metal=None, padding=10):
    """Wave-port S-parameters, post_processor.py:226-233 and :282-288.
    Returns (freq_GHz, [S11, S21]) over the trusted band."""
    d, c = parse_dat(data), parse_dat(clear)
    m = parse_dat(metal) if metal else None
    n = (padding + 1) * d["steps"]
    freq, l, h = _band(d, n)
    S = []
    for i in range(len(d["waves"])):
        F0, F1 = _fft(d["waves"][i], padding), _fft(c["waves"][i], padding)
        F2 = _fft(m["waves"][i], padding) if m else np.zeros(n)
        if i == 0:
            S.append(-1 * (F0 - F1) / (F2 - F1))
        else:
            S.append(-1 * (F0 - F2) / (F1 - F2))
    return freq[l:h + 1] / 1e9, [s[l:h + 1] for s in S]


def antenna_sparams(data, padding=10):
    """Self S-parameter of the driven port, post_processor.py:251-255."""
    d = parse_dat(data)
    n = (padding + 1) * d["steps"]
    freq, l, h = _band(d, n)
    inc = _fft(d["inc"], padding)
    V = _fft(d["ports"][0], padding)
    return freq[l:h + 1] / 1e9, [((V - inc) / inc)[l:h + 1]]


def antenna_gain(data, padding=10, imped_free=376.730313):
    """Realised gain per far-field angle and polarisation of a driven
    lumped port (post_processor.py:264-266 and :365-373): returns
    (freq_GHz, [complex columns]) whose |.|^2 is the gain and whose angle is
    the phase the CSV writes."""
    d = parse_dat(data)
    n = (padding + 1) * d["steps"]
    freq, l, h = _band(d, n)
    inc = _fft(d["inc"], padding)[l:h + 1]
    p_ant = np.abs(inc) ** 2 / (2 * d["imped"][0])
    f = freq[l:h + 1]
    out = []
    for i in range(2 * d["num_angles"]):
        s = _fft(d["ff"][i], padding)[l:h + 1]
        mag = np.sqrt(4 * np.pi * np.abs(s) ** 2 / (2 * imped_free * p_ant))
        ph = np.angle(s * np.exp(1j * 2 * np.pi * f * d["time_corr"][i // 2] - 1j * np.pi / 2) / inc)
        out.append(mag * np.exp(1j * ph))
    return f / 1e9, out


def scattering(data, clear, padding=10, full_clear=None):
    """Monostatic/bistatic RCS fields, post_processor.py:237-249; the
    phase-centre incident comes from the full clear run when the problem
    has an image plane (post_processor.py:136-143)."""
    d, c = parse_dat(data), parse_dat(clear)
    n = (padding + 1) * d["steps"]
    freq, l, h = _band(d, n)
    inc = _fft(parse_dat(full_clear)["inc_ff_pc"] if full_clear else c["inc_ff_pc"], padding)
    out = []
    for i in range(2 * d["num_angles"]):
        t = i // 2
        nph = np.exp(1j * 2 * np.pi * freq * d["time_corr"][t] - 1j * np.pi / 2)
        cph = np.exp(1j * 2 * np.pi * freq * c["time_corr"][t] - 1j * np.pi / 2)
        out.append(((_fft(d["ff"][i], padding) * nph - _fft(c["ff"][i], padding) * cph) / inc)[l:h + 1])
    return freq[l:h + 1] / 1e9, out


def csv_complex(path):
    """Golden CSV -> (freq_GHz, [complex columns]) from (dB, rad) pairs;
    RCS columns carry +10log10(4 pi) (post_processor.py:352-353)."""
    a = np.loadtxt(path, delimiter=",", skiprows=1)
    with open(path) as f:
        rcs = "dBsm" in f.readline()
    cols = []
    for q in range((a.shape[1] - 1) // 2):
        db = a[:, 1 + 2 * q] - (10 * np.log10(4 * np.pi) if rcs else 0.0)
        cols.append(10 ** (db / 20) * np.exp(1j * a[:, 2 + 2 * q]))
    return a[:, 0], cols


def match_rows(freq_ref, freq, cols):
    """Pick the rows of (freq, cols) at the reference's (possibly thinned) frequencies."""
    idx = np.clip(np.searchsorted(freq, freq_ref), 1, len(freq) - 1)
    idx = np.where(np.abs(freq[idx - 1] - freq_ref) < np.abs(freq[idx] - freq_ref), idx - 1, idx)
    # the .dat holds dt to 10 significant digits, so the grids agree to ~1e-8 relative
    assert np.max(np.abs(freq[idx] - freq_ref) / np.maximum(np.abs(freq_ref), 1e-3)) < 1e-6, "frequency grids differ"
    return [c[idx] for c in cols]
