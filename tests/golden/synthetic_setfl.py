"""Seeded synthetic potential files for the reader pins: smooth functions written in the
layouts the reference's loaders accept (``get_potential.py:58-257``). The same bytes are
written every time, so the node arrays read from them can be compared with fixtures made
by the reference's own loader.

* ``synth3.eam.alloy``: three elements, one value per line (the alloy loader reads its
  blocks with ``np.loadtxt(max_rows=...)``);
* ``synth1.eam.alloy.txt``: one element, one value per line;
* ``synth1.eam.fs.txt``: one element in the Finnis-Sinclair layout the single-element
  loader accepts: five values per line, with the innermost 167 nodes of rho(r) and
  r*phi(r) filled with 1e12 as in the Mendelev Cu file.
"""

import os

import numpy as np

N_RHO, N_R = 500, 500
D_RHO, D_R = 0.01, 0.012
FS_FILL_NODES = 167


def _functions(rng, n_el):
    r = np.arange(N_R) * D_R
    rho_g = np.arange(N_RHO) * D_RHO
    emb, den = [], []
    for _ in range(n_el):
        a, b = rng.uniform(0.5, 1.5, 2)
        emb.append(-a * np.sqrt(rho_g + 1e-3) + 0.05 * b * rho_g**2)
        den.append(b * np.exp(-a * r) * (r[-1] - r) ** 2)
    pairs = []
    for _ in range(n_el * (n_el + 1) // 2):
        a, b = rng.uniform(0.5, 1.5, 2)
        pairs.append(r * (a * np.exp(-2.0 * b * (r - 2.5)) - 2.0 * np.exp(-b * (r - 2.5)))
                     * (r[-1] - r) ** 3 / r[-1] ** 3)
    return emb, den, pairs


def _header(symbols, weights):
    lines = ["synthetic potential for reader tests", "seeded, smooth functions", "units eV A",
             f"{len(symbols)} " + " ".join(symbols),
             f"{N_RHO} {D_RHO:.16e} {N_R} {D_R:.16e} {(N_R - 1) * D_R:.16e}"]
    return lines


def _numbers(values, per_line):
    vals = [f"{v:.16e}" for v in values]
    return [" ".join(vals[k:k + per_line]) for k in range(0, len(vals), per_line)]


def write_all(directory):
    """Write the three files into ``directory``; return their paths by name."""
    out = {}
    rng = np.random.RandomState(31337)
    symbols, weights = ["Aa", "Bb", "Cc"], [10.0, 20.0, 30.0]
    emb, den, pairs = _functions(rng, 3)
    lines = _header(symbols, weights)
    for k in range(3):
        lines.append(f"{k + 1} {weights[k]:.16e} {3.5 + 0.1 * k:.16e} fcc")
        lines += _numbers(emb[k], 1) + _numbers(den[k], 1)
    for p in pairs:
        lines += _numbers(p, 1)
    out["synth3.eam.alloy"] = lines
    emb, den, pairs = _functions(rng, 1)
    lines = _header(["Dd"], [40.0])
    lines.append(f"29 {40.0:.16e} {3.6:.16e} fcc")
    lines += _numbers(emb[0], 1) + _numbers(den[0], 1) + _numbers(pairs[0], 1)
    out["synth1.eam.alloy.txt"] = lines
    emb, den, pairs = _functions(rng, 1)
    den[0][:FS_FILL_NODES] = 1e12
    pairs[0][:FS_FILL_NODES] = 1e12
    lines = _header(["Ee"], [50.0])
    lines.append(f"29 {50.0:.16e} {3.6:.16e} fcc")
    lines += _numbers(emb[0], 5) + _numbers(den[0], 5) + _numbers(pairs[0], 5)
    out["synth1.eam.fs.txt"] = lines
    paths = {}
    for name, lines in out.items():
        p = os.path.join(directory, name)
        with open(p, "w") as fh:
            fh.write("\n".join(lines) + "\n")
        paths[name] = p
    return paths
