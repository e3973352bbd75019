"""Port post-processing on the host in FP64: probe files, DFT, incident and
reflected waves, S11 and input impedance.

Restates the reference's host-side steps after a solve:
  * probe time stamps and the probe text file (scripts/lib/sim-engine.mjs:683-720):
    sample s of a probe sampled every `interval` steps sits at
    t = (s+1)*interval*dT, plus dT/2 for current (dual-grid) probes;
  * parseProbe (src/analysis.mjs:150-160);
  * dftTime2Freq (src/analysis.mjs:43-62): X(f) = sum_n x_n exp(-j 2 pi f t_n) w_n
    with w_n = t_n - t_{n-1} (w_0 = t_1 - t_0), or 1 for periodic signals;
  * Port.calcPort (src/ports.mjs:154-201): total U/I summed over a port's
    probes, incident/reflected split against Z_ref and the three powers;
  * computeS11 (scripts/lib/post-process.mjs:58-124): nf points from 0 to fmax
    (Nyquist of the voltage sampling by default), Z = U/I, Gamma = (Z-50)/(Z+50),
    S11 = 20 log10 max(|Gamma|, 1e-15), the deepest dip above DC and the
    frequency where Z is closest to 50 + 0j.
Sums run as numpy reductions (a different summation order than the
reference's loops; FP64 either way).
"""
import math

import numpy as np


def probe_times(probe, num_samples, interval, dT):
    """Sample times of a probe's ring samples (sim-engine.mjs:686-692)."""
    s = np.arange(num_samples, dtype=np.float64)
    half = 0.5 if probe.get("type") == 1 else 0.0
    return ((s + 1) * interval + half) * dT


def js_number(x):
    """A float as JavaScript's Number.prototype.toString writes it (the probe
    files are written with template literals): the shortest round-trip
    digits, positional notation for 1e-7 <= |x| < 1e21, else d.ddde+-x."""
    x = float(x)
    if x == 0.0:
        return "0"
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "Infinity" if x > 0 else "-Infinity"
    r = repr(abs(x))
    mant, _, ex = r.partition("e")
    digits, _, frac = mant.partition(".")
    e = int(ex) if ex else 0
    ds = (digits + frac).lstrip("0") or "0"
    # exponent of the leading digit: abs(x) = 0.d1d2... * 10^n
    if ex:
        n = e + len(digits)
    elif digits != "0":
        n = len(digits)
    else:
        n = -(len(frac) - len(frac.lstrip("0")))
    ds = ds.rstrip("0") or "0"
    k = len(ds)
    sign = "-" if x < 0 else ""
    if k <= n <= 21:
        return sign + ds + "0" * (n - k)
    if 0 < n <= 21:
        return sign + ds[:n] + "." + ds[n:]
    if -6 < n <= 0:
        return sign + "0." + "0" * (-n) + ds
    e1 = n - 1
    es = ("+" if e1 >= 0 else "-") + str(abs(e1))
    return sign + ds[0] + ("." + ds[1:] if k > 1 else "") + "e" + es


def probe_file(probe, times, values):
    """Text of a probe file as the reference writes it (sim-engine.mjs:711-720)."""
    kind = "voltage" if probe.get("type") == 0 else "current"
    out = ["%% time-domain %s integration by openEMS (WebGPU)\n" % kind, "%% t/s\t%s\n" % kind]
    out += ["%s\t%s\n" % (js_number(t), js_number(v)) for t, v in zip(times, values)]
    return "".join(out)


def parse_probe(text):
    """(time, values) of a probe file, comment lines skipped (analysis.mjs:150-160)."""
    t, v = [], []
    for line in text.split("\n"):
        if line.startswith("%") or not line.strip():
            continue
        p = line.split()
        t.append(float(p[0]))
        v.append(float(p[1]))
    return np.asarray(t, np.float64), np.asarray(v, np.float64)


def dft_time2freq(time, values, freq, periodic=False):
    """(re, im) of sum_n x_n exp(-j omega t_n) w_n at each frequency (analysis.mjs:43-62)."""
    time = np.asarray(time, np.float64)
    values = np.asarray(values, np.float64)
    freq = np.asarray(freq, np.float64)
    N = time.size
    if periodic:
        w = np.ones(N)
    else:
        w = np.empty(N)
        if N > 1:
            w[1:] = np.diff(time)
            w[0] = time[1] - time[0]
        elif N == 1:
            w[0] = 1.0
    ph = 2 * math.pi * np.outer(freq, time)
    xw = values * w
    return (np.cos(ph) * xw).sum(axis=1), -(np.sin(ph) * xw).sum(axis=1)


def calc_port(u_series, i_series, freq, z_ref):
    """Port.calcPort (ports.mjs:154-201).  u_series / i_series: lists of
    (time, values) for the port's voltage and current probes."""
    if not z_ref or z_ref <= 0:
        raise ValueError("Port Z_ref must be positive (got %r)" % (z_ref,))
    nf = len(freq)
    uf = np.zeros(nf, complex)
    itot = np.zeros(nf, complex)
    for t, v in u_series:
        re, im = dft_time2freq(t, v, freq)
        uf += re + 1j * im
    for t, v in i_series:
        re, im = dft_time2freq(t, v, freq)
        itot += re + 1j * im
    Z = float(z_ref)
    u_inc = 0.5 * (uf + itot * Z)
    i_inc = 0.5 * (itot + uf / Z)
    u_ref = uf - u_inc
    i_ref = i_inc - itot
    p = lambda u, i: 0.5 * (u.real * i.real + u.imag * i.imag)
    return {"uf_tot": uf, "if_tot": itot, "uf_inc": u_inc, "uf_ref": u_ref, "if_inc": i_inc, "if_ref": i_ref,
            "P_inc": p(u_inc, i_inc), "P_ref": p(u_ref, i_ref), "P_acc": p(uf, itot)}


def compute_s11(ut, it, fmax=0.0, nf=201, z0=50.0):
    """computeS11 (post-process.mjs:58-124) from (time, values) of one voltage
    and one current probe; None when either has fewer than 10 samples."""
    (tu, vu), (ti, vi) = ut, it
    if len(tu) < 10:
        return None
    dt = tu[1] - tu[0]
    fm = fmax if fmax > 0 else 0.5 / dt
    freq = np.arange(nf, dtype=np.float64) / (nf - 1) * fm
    ur, ui = dft_time2freq(tu, vu, freq)
    ir, ii = dft_time2freq(ti, vi, freq)
    denom = ir * ir + ii * ii
    ok = denom >= 1e-30
    with np.errstate(divide="ignore", invalid="ignore"):
        zr = np.where(ok, (ur * ir + ui * ii) / denom, 0.0)
        zi = np.where(ok, (ui * ir - ur * ii) / denom, 0.0)
        gdr, gdi = zr + z0, zi
        gd2 = gdr * gdr + gdi * gdi
        gnr = zr - z0
        gr = (gnr * gdr + zi * gdi) / gd2
        gi = (zi * gdr - gnr * gdi) / gd2
        s11 = np.where(ok, 20 * np.log10(np.maximum(np.sqrt(gr * gr + gi * gi), 1e-15)), 0.0)
    best = 1 + int(np.argmin(s11[1:])) if nf > 1 and s11[1:].min() < 0 else 1
    dist = np.sqrt((zr[1:] - 50) ** 2 + zi[1:] ** 2)
    dist[~np.isfinite(dist)] = np.inf
    bz = 1 + int(np.argmin(dist)) if nf > 1 else 1
    return {"freqGHz": freq / 1e9, "s11_dB": s11, "zRe": zr, "zIm": zi,
            "bestS11": float(min(0.0, s11[1:].min())) if nf > 1 else 0.0, "bestFreqGHz": float(freq[best] / 1e9),
            "bestZFreqGHz": float(freq[bz] / 1e9), "bestZRe": float(zr[bz]), "bestZIm": float(zi[bz])}
