"""Comparison helpers shared by the GPU parity tests."""
import dataclasses

import numpy as np


def with_reference_norms(cfg, init):
    """``cfg`` with every kinetic species' moment normalisation (PartSpecies::Nc) taken from the
    header of a reference state file, as an integration of the reference passes it to the C ABI;
    the reference integrates the counter-beam density numerically (VDFHelper.h:47-70)."""
    kin = [dataclasses.replace(k, norm=float(n)) for k, n in zip(cfg.kinetic, init["moment_norm"])]
    return cfg.replace(kinetic=kin)


def rel_err(a, b):
    """max |a - b| / max |b| (max-norm relative error); 0 when both are zero."""
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    scale = np.nanmax(np.abs(b)) if b.size else 0.0
    d = np.nanmax(np.abs(a - b)) if b.size else 0.0
    if scale == 0:
        return float(d)
    return float(d / scale)


def by_pid(p):
    """Particle arrays reordered by upload index."""
    order = np.argsort(p["pid"], kind="stable")
    return {k: np.asarray(v)[order] for k, v in p.items()}


def attach_pid(ref, init):
    """A reference state (tests/golden/state_io.read_state) with every particle's "pid" set to its
    index in the initial state ``init`` it was advanced from (the upload index the C ABI reports),
    found through the reference's particle ids; returns ``ref``."""
    for p, p0 in zip(ref["particles"], init["particles"]):
        id0 = np.asarray(p0["id"])
        order = np.argsort(id0, kind="stable")
        k = np.searchsorted(id0[order], p["id"])
        if not np.array_equal(id0[order][np.minimum(k, id0.size - 1)], p["id"]):
            raise ValueError("reference state holds particle ids the initial state does not")
        p["pid"] = order[k]
    return ref


def cell_keys(q1, Nx):
    return np.floor(np.asarray(q1) + 0.5 * Nx)


def state_errors(g, c, cfg, interior_only=False):
    """Relative errors of every array of two states (dicts as returned by Run.state())."""
    P = 3
    sl = slice(P, P + cfg.Nx) if interior_only else slice(None)
    errs = {}
    for key in ("B", "E", "charge", "current"):
        errs[key] = rel_err(np.asarray(g[key])[sl], np.asarray(c[key])[sl])
    for s in range(len(cfg.kinetic)):
        for key in ("n", "nV", "nvv"):
            errs[f"moments[{s}].{key}"] = rel_err(g["moments"][s][key][sl], c["moments"][s][key][sl])
        pg, pc = by_pid(g["particles"][s]), by_pid(c["particles"][s])
        for key in ("q1", "vx", "vy", "vz", "w", "real_f", "marker"):
            if key in pg and key in pc:  # real_f / marker: species whose weights evolve
                errs[f"particles[{s}].{key}"] = rel_err(pg[key], pc[key])
    for i in range(len(cfg.cold)):
        for key in ("n", "nV", "nvv", "nV_full"):
            errs[f"cold[{i}].{key}"] = rel_err(g["cold"][i][key][sl], c["cold"][i][key][sl])
    return errs


def cell_mismatches(g, c, cfg):
    """Particles whose full-grid cell differs between two states, with their distance to the
    nearest cell boundary (a tie is a mismatch closer than 1e-12)."""
    out = []
    for s in range(len(cfg.kinetic)):
        pg, pc = by_pid(g["particles"][s]), by_pid(c["particles"][s])
        kg, kc = cell_keys(pg["q1"], cfg.Nx), cell_keys(pc["q1"], cfg.Nx)
        bad = np.nonzero(kg != kc)[0]
        for i in bad:
            x = pc["q1"][i] + 0.5 * cfg.Nx
            out.append((s, int(i), float(abs(x - np.round(x)))))
    return out
