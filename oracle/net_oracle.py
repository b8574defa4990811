"""CPU oracle of the learned preconditioner network (test infrastructure only).

The network has no counterpart in the reference; this file restates, in
numpy, the forward pass, the loss and the hand-derived backward pass that the
GPU kernels (icarat2_b200/csrc/net.cu) implement, so that the GPU gradients
can be checked against it.  Only tests import it.

Network: 3-D U-net on the node grid zero-padded to multiples of 8.
  input  4 channels: residual x, y, z (divided by its L2 norm over free DOFs) and
         the node density (mean of the adjacent element densities)
  level 0  conv3(4->16)  relu  conv3(16->16) relu = S0
  level 1  pool2  conv3(16->32) relu conv3(32->32) relu = S1
  level 2  pool2  conv3(32->64) relu conv3(64->64) relu = S2
  level 3  pool2  conv3(64->128) relu conv3(128->128) relu = B3
  up2(B3) ++ S2 -> conv3(192->64) relu conv3(64->64) relu = D2
  up2(D2) ++ S1 -> conv3(96->32)  relu conv3(32->32) relu = D1
  up2(D1) ++ S0 -> conv3(48->16)  relu conv3(16->16) relu = D0
  head   conv1(16->3) + bias (FP32 output)
conv3: 3x3x3, zero padding, bias; pool2: 2x2x2 mean; up2: nearest; "++"
concatenates channels (upsampled first).  Weights and activations are stored
in BF16 (round to nearest even) and accumulated in FP32, as on the GPU
(bf16=False turns the rounding off, for finite-difference checks).
Input scale s = ||f|| (L2 over free DOFs: a point load becomes a unit spike).
Loss (scale-free, as both uses of the net are: the flexible-CG step cancels
the scale of z and the initial guess is rescaled): 1 - cos^2(y, t) over the
free DOFs, t = u / s, plus NORM_PENALTY (|y|^2 - 1)^2 to keep the free
output scale near 1.
"""
import numpy as np

NORM_PENALTY = 1e-2

LAYERS = [  # (cin, cout, kernel)
    (4, 16, 3), (16, 16, 3), (16, 32, 3), (32, 32, 3), (32, 64, 3), (64, 64, 3),
    (64, 128, 3), (128, 128, 3), (192, 64, 3), (64, 64, 3), (96, 32, 3), (32, 32, 3),
    (48, 16, 3), (16, 16, 3), (16, 3, 1)]


def n_params():
    return sum(co * ci * k ** 3 + co for ci, co, k in LAYERS)


def unpack(w):
    """flat parameter vector -> list of (W[co][ci][k^3], b[co])"""
    out, o = [], 0
    for ci, co, k in LAYERS:
        nw = co * ci * k ** 3
        W = w[o:o + nw].reshape(co, ci, k ** 3)
        o += nw
        b = w[o:o + co]
        o += co
        out.append((W, b))
    return out


def bf16(a):
    """round float32 values to bfloat16 (nearest even), returned as float32"""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def padded(n):
    return (n + 7) // 8 * 8


def conv3(x, W, b, dt):
    """x[ci][z][y][x], W[co][ci][27] -> y[co][...] (3x3x3, zero padding)"""
    ci, Z, Y, X = x.shape
    xp = np.zeros((ci, Z + 2, Y + 2, X + 2), dtype=dt)
    xp[:, 1:-1, 1:-1, 1:-1] = x
    y = np.zeros((W.shape[0], Z, Y, X), dtype=dt)
    for tap in range(27):
        dz, dy, dx = tap // 9, (tap // 3) % 3, tap % 3
        sl = xp[:, dz:dz + Z, dy:dy + Y, dx:dx + X]
        y += np.einsum("oc,czyx->ozyx", W[:, :, tap].astype(dt), sl)
    return y + b.astype(dt)[:, None, None, None]


def conv3_back(x, W, dy, dt):
    """gradients of conv3: dx, dW, db"""
    ci, Z, Y, X = x.shape
    xp = np.zeros((ci, Z + 2, Y + 2, X + 2), dtype=dt)
    xp[:, 1:-1, 1:-1, 1:-1] = x
    dxp = np.zeros_like(xp)
    dW = np.zeros(W.shape, dtype=dt)
    for tap in range(27):
        dz, dyy, dx = tap // 9, (tap // 3) % 3, tap % 3
        sl = xp[:, dz:dz + Z, dyy:dyy + Y, dx:dx + X]
        dW[:, :, tap] = np.einsum("ozyx,czyx->oc", dy, sl)
        dxp[:, dz:dz + Z, dyy:dyy + Y, dx:dx + X] += np.einsum("oc,ozyx->czyx",
                                                               W[:, :, tap].astype(dt), dy)
    return dxp[:, 1:-1, 1:-1, 1:-1], dW, dy.sum(axis=(1, 2, 3))


def pool(x):
    c, Z, Y, X = x.shape
    return x.reshape(c, Z // 2, 2, Y // 2, 2, X // 2, 2).mean(axis=(2, 4, 6))


def pool_back(d):
    return up(d) / 8.0


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)


def up_back(d):
    c, Z, Y, X = d.shape
    return d.reshape(c, Z // 2, 2, Y // 2, 2, X // 2, 2).sum(axis=(2, 4, 6))


def inputs(nx, ny, nz, rho, f, fix):
    """input tensor [4][Pz][Py][Px] and the scale s; f and fix are node-major
    arrays [nz+1][ny+1][nx+1][3] (fix: bool per component)"""
    NX, NY, NZ = nx + 1, ny + 1, nz + 1
    P = (padded(NZ), padded(NY), padded(NX))
    free = ~fix
    s = np.sqrt((f[free] ** 2).sum()) if free.any() else 1.0
    s = s if s > 0 else 1.0
    x = np.zeros((4,) + P, dtype=np.float32)
    for c in range(3):
        x[c, :NZ, :NY, :NX] = np.where(free[..., c], f[..., c] / s, 0.0)
    r = rho.reshape(nz, ny, nx)
    rp = np.zeros((nz + 2, ny + 2, nx + 2))
    cnt = np.zeros_like(rp)
    rp[1:-1, 1:-1, 1:-1] = r
    cnt[1:-1, 1:-1, 1:-1] = 1.0
    acc = np.zeros((NZ, NY, NX))
    nacc = np.zeros((NZ, NY, NX))
    for dz in range(2):
        for dy in range(2):
            for dx in range(2):
                acc += rp[dz:dz + NZ, dy:dy + NY, dx:dx + NX]
                nacc += cnt[dz:dz + NZ, dy:dy + NY, dx:dx + NX]
    x[3, :NZ, :NY, :NX] = acc / nacc
    return x, s


def forward(w, xin, bf=True):
    """returns the head output [3][...] and the saved activations"""
    dt = np.float32 if bf else np.float64
    rd = bf16 if bf else (lambda a: a)
    P = [(rd(W.astype(np.float32)) if bf else W.astype(np.float64), b) for W, b in unpack(w)]
    act = {}

    def cr(name, x, i):
        y = np.maximum(conv3(x, P[i][0], P[i][1], dt), 0.0)
        act[name] = rd(y).astype(dt)
        return act[name]

    x = rd(xin).astype(dt)
    act["in"] = x
    a0 = cr("a0", x, 0)
    s0 = cr("s0", a0, 1)
    p1 = rd(pool(s0)).astype(dt)
    act["p1"] = p1
    a1 = cr("a1", p1, 2)
    s1 = cr("s1", a1, 3)
    p2 = rd(pool(s1)).astype(dt)
    act["p2"] = p2
    a2 = cr("a2", p2, 4)
    s2 = cr("s2", a2, 5)
    p3 = rd(pool(s2)).astype(dt)
    act["p3"] = p3
    a3 = cr("a3", p3, 6)
    b3 = cr("b3", a3, 7)
    c2 = np.concatenate([up(b3), s2])
    act["c2"] = c2
    e2 = cr("e2", c2, 8)
    d2 = cr("d2", e2, 9)
    c1 = np.concatenate([up(d2), s1])
    act["c1"] = c1
    e1 = cr("e1", c1, 10)
    d1 = cr("d1", e1, 11)
    c0 = np.concatenate([up(d1), s0])
    act["c0"] = c0
    e0 = cr("e0", c0, 12)
    d0 = cr("d0", e0, 13)
    Wh, bh = P[14]
    out = np.einsum("oc,czyx->ozyx", Wh[:, :, 0].astype(dt), d0) + \
        bh.astype(dt)[:, None, None, None]
    return out, act, P


def loss_and_grads(w, xin, target, mask, bf=True):
    """1 - cos^2(out, target) over mask (target, mask: [3][...]) and the
    gradient of the flat parameter vector"""
    dt = np.float32 if bf else np.float64
    out, act, P = forward(w, xin, bf)
    y = np.where(mask, out, 0.0).astype(np.float64)
    t = np.where(mask, target, 0.0).astype(np.float64)
    A, Y, T = float((y * t).sum()), float((y * y).sum()) + 1e-30, float((t * t).sum())
    loss = 1.0 - A * A / (Y * T) + NORM_PENALTY * (Y - 1.0) ** 2
    dout = np.where(mask, -2.0 * A / (Y * T) * t +
                    (2.0 * A * A / (Y * Y * T) + 4.0 * NORM_PENALTY * (Y - 1.0)) * y,
                    0.0).astype(dt)
    grads = [None] * len(LAYERS)
    Wh = P[14][0]
    grads[14] = (np.einsum("ozyx,czyx->oc", dout, act["d0"])[:, :, None],
                 dout.sum(axis=(1, 2, 3)))
    dd0 = np.einsum("oc,ozyx->czyx", Wh[:, :, 0].astype(dt), dout)

    def back(dy_post, y_post, x_in, i):
        dy = np.where(y_post > 0, dy_post, 0.0).astype(dt)
        dx, dW, db = conv3_back(x_in, P[i][0], dy, dt)
        grads[i] = (dW, db)
        return dx

    de0 = back(dd0, act["d0"], act["e0"], 13)
    dc0 = back(de0, act["e0"], act["c0"], 12)
    dd1 = up_back(dc0[:32])
    ds0 = dc0[32:]
    de1 = back(dd1, act["d1"], act["e1"], 11)
    dc1 = back(de1, act["e1"], act["c1"], 10)
    dd2 = up_back(dc1[:64])
    ds1 = dc1[64:]
    de2 = back(dd2, act["d2"], act["e2"], 9)
    dc2 = back(de2, act["e2"], act["c2"], 8)
    db3 = up_back(dc2[:128])
    ds2 = dc2[128:]
    da3 = back(db3, act["b3"], act["a3"], 7)
    dp3 = back(da3, act["a3"], act["p3"], 6)
    ds2 = ds2 + pool_back(dp3)
    da2 = back(ds2, act["s2"], act["a2"], 5)
    dp2 = back(da2, act["a2"], act["p2"], 4)
    ds1 = ds1 + pool_back(dp2)
    da1 = back(ds1, act["s1"], act["a1"], 3)
    dp1 = back(da1, act["a1"], act["p1"], 2)
    ds0 = ds0 + pool_back(dp1)
    da0 = back(ds0, act["s0"], act["a0"], 1)
    back(da0, act["a0"], act["in"], 0)
    flat = np.concatenate([np.concatenate([g[0].ravel(), g[1].ravel()]) for g in grads])
    return loss, flat, out
