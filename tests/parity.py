"""Parity figures shared by the GPU solver tests.

Two relative errors of a right-hand side per conserved component c:
* plain: max_points |dQ_gpu - dQ_oracle| / max_points |dQ_oracle|;
* term scale: the same difference over max(max|dQ_c|, max_d max|F_dc| / h_d),
  the size of the directional flux-divergence terms summed into dQ_c.  The
  asserted bound (1e-12) is on this figure: where the terms cancel (the energy
  equation of a Taylor-Green box sums terms of size ~250/h into an O(1)
  result) a few ulp of the terms are more than 1e-12 of the result.
Both are recorded, so the effect of the rescaling is visible in the run's
summary."""
import numpy as np

LINES = []


def rhs_errors(a, b, scales):
    """(plain, term-scale) relative errors per component of interior arrays a (device), b (oracle)."""
    plain, term = [], []
    for c in range(b.shape[0]):
        d = float(np.abs(a[c] - b[c]).max())
        m = float(np.abs(b[c]).max())
        plain.append(d / m if m > 0 else d)
        sc = max(m, scales[c])
        term.append(d / sc if sc > 0 else d)
    return plain, term


def record(label, plain=None, term=None, **extra):
    parts = [label]
    if plain is not None:
        parts.append("plain " + " ".join(f"{e:.1e}" for e in plain))
    if term is not None:
        parts.append("term-scale " + " ".join(f"{e:.1e}" for e in term))
    parts += [f"{k} {v:.2e}" if isinstance(v, float) else f"{k} {v}" for k, v in extra.items()]
    LINES.append(" | ".join(parts))
