"""Phase-function CDFs with awkward shapes for the scattering tests."""
import numpy as np


def odd_phase_cdfs(nB, nA, seed):
    """Phase CDFs with flat stretches (angle ranges of zero probability), a
    single jump, a forward spike with a long thin tail, and a backward ramp."""
    rng = np.random.default_rng(seed)
    cdf = np.zeros((nB, nA))
    for b in range(nB):
        kind = b % 4
        pdf = np.zeros(nA - 1)
        if kind == 0:
            pdf[rng.choice(nA - 1, 5, replace=False)] = rng.random(5) + 0.1
        elif kind == 1:
            pdf[rng.integers(0, nA - 1)] = 1.0
        elif kind == 2:
            pdf[:] = 1e-4
            pdf[0] = 1.0
        else:
            pdf[nA // 2:] = np.linspace(0.0, 1.0, nA - 1 - nA // 2)
        c = np.concatenate([[0.0], np.cumsum(pdf)])
        cdf[b] = c / c[-1]
    cdf = cdf.astype(np.float32)
    cdf[:, -1] = 1.0
    return cdf
