"""Inputs for the Green-operator tests: a cubic reference medium and a compatible strain field."""
import numpy as np

IJV = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]


def cubic_c4(c11=250000.0, c12=150000.0, c44=120000.0):
    c66 = np.zeros((6, 6))
    c66[:3, :3] = c12
    np.fill_diagonal(c66[:3, :3], c11)
    c66[3, 3] = c66[4, 4] = c66[5, 5] = c44
    c4 = np.zeros((3, 3, 3, 3))
    for i, (a, b) in enumerate(IJV):
        for j, (c, d) in enumerate(IJV):
            for (p, q) in ((a, b), (b, a)):
                for (r, s) in ((c, d), (d, c)):
                    c4[p, q, r, s] = c66[i, j]
    return c4


def medium(orc, scale=2.0):
    """c0 = scale * cubic stiffness and s0 = its compliance (b-basis inverse), like calc_c0's xc0 scaling."""
    c0 = scale * cubic_c4()
    s0 = orc.chg_b66_to_t4(np.linalg.inv(orc.chg_t4_to_b66(c0)))
    return c0, s0


def compatible_field(shape, c0, modes=((1, 2, -1), (0, 3, 2)), seed=0):
    """tau = c0 : grad(u) for a smooth periodic displacement u built from a few Fourier modes
    (no DC, no Nyquist content); the Green operator maps it to -grad(u)."""
    n1, n2, n3 = shape
    rng = np.random.default_rng(seed)
    x = np.stack(np.meshgrid(np.arange(n1), np.arange(n2), np.arange(n3), indexing="ij"), axis=-1).astype(float)
    G = np.zeros((n1, n2, n3, 3, 3))
    for m in modes:
        xi = 2.0 * np.pi * np.array(m) / np.array([n1, n2, n3])
        a = rng.standard_normal(3)
        ph = x @ xi
        # u = a cos(xi.x)  ->  du_k/dx_l = -a_k xi_l sin(xi.x)
        G += -np.einsum("k,l,...->...kl", a, xi, np.sin(ph))
    tau = np.einsum("klmn,...mn->...kl", c0, G)
    to_soa = lambda t: np.ascontiguousarray(np.transpose(t, (3, 4, 2, 1, 0)).reshape(9, -1))
    return to_soa(tau), to_soa(G)
