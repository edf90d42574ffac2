"""The wall model's Newton exits (csrc/physics.cuh spalding_utau): stopping at an exact fixed
point, or at a two-cycle with the last iterate chosen by the parity of the steps left,
returns what all n_iter steps of the reference's safeguarded Newton return
(wmles/wall_model.py:19-40).  The device code's exits restated here in NumPy scalar
arithmetic and checked against the full iteration on the CPU."""
import numpy as np

KAPPA, B = 0.41, 5.2
EKB = np.exp(-KAPPA * B)


def _g(up, Reh):
    ku = KAPPA * up
    ex = np.exp(ku)
    F = up + EKB * (ex - 1.0 - ku - 0.5 * ku * ku - ku * ku * ku / 6.0) - Reh / up
    dF = 1.0 + EKB * KAPPA * (ex - 1.0 - ku - 0.5 * ku * ku) + Reh / (up * up)
    return min(max(up - F / dF, 0.5 * up), 100.0)


def _full(Reh, n):
    up, last = min(max(np.sqrt(Reh), 1.0), 25.0), 0.0
    for _ in range(n):
        nx = _g(up, Reh)
        last, up = nx - up, nx
    return up, not (abs(last) <= 1e-8 * up)


def _with_exits(Reh, n):
    up = min(max(np.sqrt(Reh), 1.0), 25.0)
    last, prev = 0.0, up
    for it in range(n):
        nx = _g(up, Reh)
        if nx == up:
            return up, False, it
        if it > 0 and nx == prev:
            fin = nx if (n - it + 1) % 2 == 0 else up
            return fin, not (abs(nx - up) <= 1e-8 * fin), it
        last, prev, up = nx - up, up, nx
    return up, not (abs(last) <= 1e-8 * up), n


def test_exits_return_the_full_iteration():
    rng = np.random.default_rng(3)
    Rehs = np.concatenate([10 ** rng.uniform(-1, 6, 3000), [1e-3, 1.0, 625.0, 1e7]])
    cycles = 0
    for n in (30, 29, 4, 1):
        for Reh in Rehs:
            fin, moving, it = _with_exits(Reh, n)
            assert (fin, moving) == _full(Reh, n), (Reh, n)
            if n == 30 and it < n and _g(_g(fin, Reh), Reh) == fin and _g(fin, Reh) != fin:
                cycles += 1
    assert cycles > 0          # the two-cycle exit is exercised, not only the fixed point
