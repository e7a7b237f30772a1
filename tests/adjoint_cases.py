"""Geometries for the adjoint tests: non-uniform steps across interfaces (hx differs across an x interface,
hy across a y interface), Neumann and periodic faces."""
import types

D, N, P = 0, 1, 2


def skewed_t():
    """A (centre) with B at A's x+ face (different hx) and C at A's y+ face (different hy)."""
    return types.SimpleNamespace(
        nx=[12, 20, 12], ny=[10, 10, 14], hx=[1 / 12, 1 / 40, 1 / 12], hy=[1 / 10, 1 / 10, 1 / 35],
        bc=[[D, D, D, D], [D, N, D, D], [D, D, D, N]], connections=[(0, 1, 1), (0, 3, 2)])


def periodic_arm():
    """A with B at its x- face; B is periodic in y (both y faces outer), A Neumann at the far x face."""
    return types.SimpleNamespace(
        nx=[16, 10], ny=[12, 12], hx=[1 / 16, 1 / 30], hy=[1 / 12, 1 / 12],
        bc=[[D, N, D, D], [D, D, P, P]], connections=[(0, 0, 1)])


CASES = {"skewed_t": skewed_t, "periodic_arm": periodic_arm}
