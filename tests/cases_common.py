"""Shared case definitions for the tests (boundary-condition combinations,
grids and boundary values)."""
import numpy as np

# Every (u.left,u.right,u.low,u.up, v.left,v.right,v.low,v.up) combination
# the reference's BC checks allow and its mesh code covers
# (boundary_conditions.m:17-40, operator_mesh.m:185-320), as named cases.
BC_COMBOS = {
    "cavity": dict(u=dict(left="dir", right="dir", low="dir", up="dir"),
                   v=dict(left="dir", right="dir", low="dir", up="dir")),
    "periodic": dict(u=dict(left="per", right="per", low="per", up="per"),
                     v=dict(left="per", right="per", low="per", up="per")),
    "channel": dict(u=dict(left="dir", right="pres", low="dir", up="dir"),
                    v=dict(left="dir", right="sym", low="dir", up="dir")),
    "channel_rev": dict(u=dict(left="pres", right="dir", low="dir", up="dir"),
                        v=dict(left="sym", right="dir", low="dir", up="dir")),
    "open_x": dict(u=dict(left="pres", right="pres", low="sym", up="sym"),
                   v=dict(left="sym", right="sym", low="dir", up="dir")),
    "per_x_walls": dict(u=dict(left="per", right="per", low="dir", up="dir"),
                        v=dict(left="per", right="per", low="dir", up="dir")),
    "per_y_open": dict(u=dict(left="dir", right="pres", low="per", up="per"),
                       v=dict(left="dir", right="sym", low="per", up="per")),
    "open_y": dict(u=dict(left="dir", right="dir", low="dir", up="dir"),
                   v=dict(left="dir", right="dir", low="dir", up="pres")),
    "open_y_both": dict(u=dict(left="sym", right="sym", low="per", up="per")  # placeholder replaced below
                        , v=dict(left="sym", right="sym", low="pres", up="pres")),
}
# u.left/right must be dir/per/pres; fix the placeholder to a legal combo:
BC_COMBOS["open_y_both"] = dict(u=dict(left="dir", right="dir", low="sym", up="sym"),
                                v=dict(left="dir", right="dir", low="pres", up="pres"))


def grid_uniform(N, a=0.0, b=1.0):
    return a + (b - a) * np.arange(N + 1) / N


def grid_stretched(N, a=0.0, b=1.0, beta=1.5):
    """tanh-clustered grid towards both ends (deterministic, non-uniform)."""
    s = np.linspace(-1.0, 1.0, N + 1)
    z = np.tanh(beta * s) / np.tanh(beta)
    return a + (b - a) * (z + 1) / 2


def is_closed(bc):
    """No outflow ('pres') boundary: the pressure matrix is singular and the
    boundary data must carry zero net normal flux for a consistent system."""
    return "pres" not in (bc["u"]["left"], bc["u"]["right"], bc["v"]["low"], bc["v"]["up"])


def smooth_bc(seed, closed=False):
    """Smooth, time-dependent boundary values (so every BC vector is non-zero).
    closed=True makes the normal components (u on left/right, v on low/up)
    zero, as a closed domain needs."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.5, 1.5, 6)

    def uBC(x, y, t):
        x = np.atleast_1d(np.asarray(x, float))
        y = np.atleast_1d(np.asarray(y, float))
        if closed and len(x) == 1 and len(y) > 1:
            return np.zeros(len(y))
        X = np.tile(x, len(y)) if len(y) > 1 else x
        Y = np.repeat(y, len(x)) if len(y) > 1 else np.full(len(x), y[0])
        return a[0] * np.sin(2 * X + a[1] * Y + t) + a[2] * 0.3

    def vBC(x, y, t):
        x = np.atleast_1d(np.asarray(x, float))
        y = np.atleast_1d(np.asarray(y, float))
        if closed and len(y) == 1 and len(x) > 1:
            return np.zeros(len(x))
        X = np.tile(x, len(y)) if len(y) > 1 else x
        Y = np.repeat(y, len(x)) if len(y) > 1 else np.full(len(x), y[0])
        return a[3] * np.cos(a[4] * X - 3 * Y + 0.5 * t) + 0.1 * a[5]

    return uBC, vBC


def unsteady_bc(seed):
    """The boundary functions of smooth_bc(seed) with their time derivatives
    (for BC_unsteady = 1 cases): returns uBC, vBC, dudtBC, dvdtBC."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.5, 1.5, 6)
    uBC, vBC = smooth_bc(seed)

    def _xy(x, y):
        x = np.atleast_1d(np.asarray(x, float))
        y = np.atleast_1d(np.asarray(y, float))
        X = np.tile(x, len(y)) if len(y) > 1 else x
        Y = np.repeat(y, len(x)) if len(y) > 1 else np.full(len(x), y[0])
        return X, Y

    def dudtBC(x, y, t):
        X, Y = _xy(x, y)
        return a[0] * np.cos(2 * X + a[1] * Y + t)

    def dvdtBC(x, y, t):
        X, Y = _xy(x, y)
        return -0.5 * a[3] * np.sin(a[4] * X - 3 * Y + 0.5 * t)

    return uBC, vBC, dudtBC, dvdtBC
