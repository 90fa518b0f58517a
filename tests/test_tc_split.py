"""The arithmetic of the tensor-core replica pass (kernel 5), emulated in numpy on the CPU.

Each FP32 operand x is split into a head (its sign, exponent and the 10 significand
bits TF32 keeps: one mask) and the exact FP32 tail x - head; the tensor core reads
TF32 operands, so it keeps 11 significant bits of the tail as well. A product a.b is
summed as ah.bh + ah.bl + al.bh (the tail.tail product is dropped). These tests pin
the error bound quoted for that scheme (under 2^-19 relative per product) and that a
site's pair contraction formed this way stays far inside the FP32 dE bar of the replay
tests (1e-5 of sum|c| (sum|znew| + sum|zold|)).
"""
import numpy as np

MASK = np.uint32(0xFFFFE000)


def head(x):
    x = np.asarray(x, np.float32)
    return (x.view(np.uint32) & MASK).view(np.float32)


def split(x):
    x = np.asarray(x, np.float32)
    h = head(x)
    t = (x - h).astype(np.float32)  # exact in FP32
    return h, head(t)  # the tensor core drops the tail's low 13 bits


def split_product(a, b):
    ah, al = split(a)
    bh, bl = split(b)
    f = lambda u: u.astype(np.float64)  # noqa: E731  (the MMA forms exact products)
    return f(ah) * f(bh) + f(ah) * f(bl) + f(al) * f(bh)


def test_head_plus_tail_is_exact_and_the_tail_is_small():
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(200_000) * 10.0 ** rng.uniform(-6, 1, 200_000)).astype(np.float32)
    h = head(x)
    t = (x - h).astype(np.float32)
    assert np.array_equal((h.astype(np.float64) + t.astype(np.float64)).astype(np.float32), x)
    nz = x != 0
    assert np.all(np.abs(t[nz]) < 2.0 ** -10 * np.abs(x[nz]))


def test_split_product_error_is_below_two_to_minus_19():
    rng = np.random.default_rng(2)
    a = (rng.standard_normal(500_000) * 10.0 ** rng.uniform(-4, 1, 500_000)).astype(np.float32)
    b = (rng.standard_normal(500_000) * 10.0 ** rng.uniform(-4, 1, 500_000)).astype(np.float32)
    exact = a.astype(np.float64) * b.astype(np.float64)
    rel = np.abs(split_product(a, b) - exact) / np.abs(exact)
    assert rel.max() < 2.0 ** -19
    # a single TF32 product (no tails) would be about 2^-10 off: the tails are what keep FP32 accuracy
    one = head(a).astype(np.float64) * head(b).astype(np.float64)
    assert (np.abs(one - exact) / np.abs(exact)).max() > 2.0 ** -12


def zrow(v):
    """Normalised real harmonics l = 1, 2 of unit vectors v (rows), in the kernel's order."""
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    n1, c2a, c20, c22 = 0.4886025119029199, 1.0925484305920792, 0.31539156525252005, 0.5462742152960396
    return np.stack([n1 * y, n1 * z, n1 * x, c2a * x * y, c2a * y * z, c20 * (3 * z * z - 1), c2a * x * z,
                     c22 * (x * x - y * y)], axis=1)


def test_site_contraction_stays_inside_the_de_bar():
    """One fcc site: 54 pair blocks of N(0, 1 meV) entries and 32 replicas. The
    coefficients c = sum_rec W_rec z_rec, accumulated in FP32 from split products in
    groups of eight records (as the MMA does), against FP64; dE = c . (znew - zold)
    must lie far inside the replay tests' 1e-5 scaled bar."""
    rng = np.random.default_rng(3)
    K, R = 54, 32
    W = (rng.standard_normal((K, 8, 8)) * 1e-3).astype(np.float32)
    v = rng.standard_normal((K, R, 3))
    v /= np.linalg.norm(v, axis=2, keepdims=True)
    Z = zrow(v.reshape(-1, 3)).reshape(K, R, 8).astype(np.float32)
    exact = np.einsum("kij,krj->ri", W.astype(np.float64), Z.astype(np.float64))
    acc = np.zeros((R, 8), np.float32)
    for g0 in range(0, K, 8):
        part = np.zeros((R, 8))
        for k in range(g0, min(g0 + 8, K)):
            for j in range(8):
                part += split_product(Z[k, :, j][:, None], W[k, :, j][None, :])
        acc = (acc + part.astype(np.float32)).astype(np.float32)
    old = rng.standard_normal((R, 3))
    new = rng.standard_normal((R, 3))
    old /= np.linalg.norm(old, axis=1, keepdims=True)
    new /= np.linalg.norm(new, axis=1, keepdims=True)
    zo, zn = zrow(old), zrow(new)
    dE_dev = np.sum(acc.astype(np.float64) * (zn - zo), axis=1)
    dE_64 = np.sum(exact * (zn - zo), axis=1)
    scale = np.abs(exact).sum(axis=1) * (np.abs(zn).sum(axis=1) + np.abs(zo).sum(axis=1))
    assert np.all(np.abs(dE_dev - dE_64) <= 1e-6 * scale)
