"""Reader for the raw state files written by oracle/ref/ref_driver.cc (``dump``).

layout (little endian):
  char[8] "H1DSTAT2" (or "H1DSTATE": no real_f/marker); int64 Nx, pad, n_kinetic, n_cold, step;
  double moment_norm[n_kinetic]
  per kinetic species: int64 n; double q1[n], vx[n], vy[n], vz[n], w[n]; int64 id[n];
                       double real_f[n], marker[n]      (the phase-space density Particle::PSD)
  B[M*3], E[M*3], charge[M], current[M*3]                       (M = Nx + 2*pad)
  per kinetic species: n[M], nV[M*3], nvv[M*6]
  per cold species:    n_full[M], nV_full[M*3], n[M], nV[M*3], nvv[M*6]
"""
import numpy as np


def read_state(path):
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] not in (b"H1DSTATE", b"H1DSTAT2"):
        raise ValueError("not a state file")
    with_psd = buf[:8] == b"H1DSTAT2"
    off = 8

    def i64(k=1):
        nonlocal off
        a = np.frombuffer(buf, dtype="<i8", count=k, offset=off)
        off += 8 * k
        return a

    def f64(k):
        nonlocal off
        a = np.frombuffer(buf, dtype="<f8", count=k, offset=off).copy()
        off += 8 * k
        return a

    Nx, pad, nk, nc, step = (int(x) for x in i64(5))
    M = Nx + 2 * pad
    st = dict(Nx=Nx, pad=pad, step=step, moment_norm=f64(nk), particles=[], moments=[], cold=[])
    for _ in range(nk):
        n = int(i64()[0])
        p = {k: f64(n) for k in ("q1", "vx", "vy", "vz", "w")}
        p["id"] = i64(n).copy()
        if with_psd:
            p["real_f"], p["marker"] = f64(n), f64(n)
        else:
            p["real_f"], p["marker"] = p["w"].copy(), np.ones(n)
        st["particles"].append(p)
    st["B"] = f64(3 * M).reshape(M, 3)
    st["E"] = f64(3 * M).reshape(M, 3)
    st["charge"] = f64(M)
    st["current"] = f64(3 * M).reshape(M, 3)
    for _ in range(nk):
        st["moments"].append(dict(n=f64(M), nV=f64(3 * M).reshape(M, 3), nvv=f64(6 * M).reshape(M, 6)))
    for _ in range(nc):
        st["cold"].append(dict(n_full=f64(M), nV_full=f64(3 * M).reshape(M, 3), n=f64(M),
                               nV=f64(3 * M).reshape(M, 3), nvv=f64(6 * M).reshape(M, 6)))
    if off != len(buf):
        raise ValueError("trailing bytes in state file")
    return st


def write_state(path, st):
    """Write a state dict (as read_state returns it) in the "H1DSTAT2" layout above."""
    nk, nc = len(st["particles"]), len(st["cold"])
    with open(path, "wb") as f:
        f.write(b"H1DSTAT2")
        np.array([st["Nx"], st["pad"], nk, nc, st["step"]], dtype="<i8").tofile(f)
        np.asarray(st["moment_norm"], dtype="<f8").tofile(f)
        for p in st["particles"]:
            np.array([p["q1"].size], dtype="<i8").tofile(f)
            for k in ("q1", "vx", "vy", "vz", "w"):
                np.asarray(p[k], dtype="<f8").tofile(f)
            np.asarray(p["id"], dtype="<i8").tofile(f)
            np.asarray(p["real_f"], dtype="<f8").tofile(f)
            np.asarray(p["marker"], dtype="<f8").tofile(f)
        for k in ("B", "E", "charge", "current"):
            np.asarray(st[k], dtype="<f8").tofile(f)
        for m in st["moments"]:
            for k in ("n", "nV", "nvv"):
                np.asarray(m[k], dtype="<f8").tofile(f)
        for c in st["cold"]:
            for k in ("n_full", "nV_full", "n", "nV", "nvv"):
                np.asarray(c[k], dtype="<f8").tofile(f)
