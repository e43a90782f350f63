"""Sampled macroscopic fields: the reference's [cell][18] layout and the
comparison of two runs' fields (mixed precision against FP64).

Layout: MacroIndex, src/ProcessDSMC.h:28-49, filled by writeAveragedMacro
(src/ProcessDSMC.cpp:3126-3181).
"""
from __future__ import annotations

import numpy as np

FIELD_NAMES = ["rho", "ux", "uy", "uz", "T", "sxx", "sxy", "syy", "syz", "szz", "szx",
               "qx", "qy", "qz", "Tr", "qrx", "qry", "qrz"]


def field_scales(m: np.ndarray) -> np.ndarray:
    """A per-cell magnitude for each field, to express differences in:
    density, speed for the velocity components, temperature, rho T for the
    stresses, rho T^1.5 for the heat fluxes, the rotational temperature."""
    m = np.asarray(m, dtype=float)
    rho = np.abs(m[:, 0])
    T = np.abs(m[:, 4])
    speed = np.linalg.norm(m[:, 1:4], axis=1)
    s = np.empty_like(m)
    s[:, 0] = rho
    s[:, 1:4] = speed[:, None]
    s[:, 4] = T
    s[:, 5:11] = (rho * T)[:, None]
    s[:, 11:14] = (rho * T ** 1.5)[:, None]
    s[:, 14] = np.abs(m[:, 14])
    s[:, 15:18] = (rho * T ** 1.5)[:, None]
    return s


def compare_windows(wa: np.ndarray, wb: np.ndarray, volume: np.ndarray) -> dict:
    """Two runs' window-averaged fields, (windows, cells, 18) each (the
    `record` fields handed to the GSIS step at every exchange), run a against
    run b. Cells that hold particles in every window of both runs count.

    Per field:
      - domain_rel: |sum_c m_c (a_c - b_c)| / sum_c m_c s_c, the
        mass-weighted domain difference relative to the field's scale s
        (m_c = volume x density of run b);
      - within_3se: the fraction of cells whose difference of the window
        means is within 3 standard errors (batch means over the windows,
        both runs' errors combined);
      - rel_noise: the median standard error of the difference relative to
        the field's scale (the resolution a per-cell comparison has).
    worst_domain_rel is the largest domain_rel over the fields."""
    wa = np.asarray(wa, dtype=float)
    wb = np.asarray(wb, dtype=float)
    nwin = wa.shape[0]
    ok = np.all(wa[:, :, 0] > 0, axis=0) & np.all(wb[:, :, 0] > 0, axis=0)
    ok &= np.all(np.isfinite(wa), axis=(0, 2)) & np.all(np.isfinite(wb), axis=(0, 2))
    ma, mb = wa[:, ok].mean(0), wb[:, ok].mean(0)
    se = np.sqrt(wa[:, ok].var(0, ddof=1) / nwin + wb[:, ok].var(0, ddof=1) / nwin) if nwin > 1 else None
    scale = field_scales(mb)
    mass = np.asarray(volume, dtype=float)[ok] * mb[:, 0]
    out = {"cells": int(ok.sum()), "windows": int(nwin), "fields": {}}
    worst = 0.0
    for k, name in enumerate(FIELD_NAMES):
        den = float(np.sum(mass * scale[:, k]))
        dom = float(abs(np.sum(mass * (ma[:, k] - mb[:, k]))) / den) if den > 0 else 0.0
        f = {"domain_rel": dom}
        if se is not None:
            good = se[:, k] > 0
            z = np.abs(ma[good, k] - mb[good, k]) / se[good, k]
            f["within_3se"] = float(np.mean(z <= 3.0)) if good.any() else 1.0
            pos = scale[:, k] > 0
            f["rel_noise"] = float(np.median(se[pos, k] / scale[pos, k])) if pos.any() else 0.0
        out["fields"][name] = f
        worst = max(worst, dom)
    out["worst_domain_rel"] = worst
    if se is not None:
        out["worst_within_3se"] = min(f["within_3se"] for f in out["fields"].values())
    return out
