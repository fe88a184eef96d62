"""CPU oracle for the learned SGS closure -- TEST INFRASTRUCTURE ONLY.

The learned closure has no counterpart in the Fortran reference: it stands in
for the dynamic procedure (``src/compute_sgs.f90:171-286``) at the same update
cadence.  This module restates the CUDA closure (``new_repo_b200/csrc/mlp.cu``)
on the CPU so that tests can check the GPU's features, forward pass and
training gradients.  Only ``tests/`` may import it.

Network: 8 features (7 resolved invariants and the coefficient before the
update, which carries the Lagrangian memory of the dynamic procedure) ->
64 (GELU) -> 64 (GELU) -> 1, output y the normalised change of log Cs^2 over
the update, ``Cs^2 = clamp(Cs^2_prev * exp(ymu + ysd * y), 1e-24, 1)`` with
Cs^2_prev floored at 1e-6.

Precision model of the GPU kernels (reproduced by ``forward``/``grad`` with
``bf16=True``):
* layer-1 and layer-2 operands are BF16 (round to nearest even): the
  normalised features x, W1, the hidden activations h1 and W2; products are
  accumulated in FP32 and the biases added in FP32;
* the output layer (w3, b3) and every elementwise step are FP32;
* backward: g2 = dy * w3 * gelu'(z2) in FP32; dW2 = h1_bf16^T g2 (FP32);
  delta1 = (bf16(g2) bf16(W2)^T) * gelu'(z1); dW1 = x_bf16^T delta1.
With ``bf16=False`` the same formulas in FP64 give the exact gradient of the
FP64 network (checked against finite differences in ``tests/test_mlp.py``).
"""
from __future__ import annotations

import numpy as np

NIN, NH = 8, 64
O_W1 = 0
O_B1 = O_W1 + NIN * NH
O_W2 = O_B1 + NH
O_B2 = O_W2 + NH * NH
O_W3 = O_B2 + NH
O_B3 = O_W3 + NH
NP = O_B3 + 1  # 4801
S_MU, S_SD, S_MIN, S_MAX, S_YMU, S_YSD, S_YMIN, S_YMAX = 0, 8, 16, 24, 32, 33, 34, 35
NS = 36
LOG_CS_FLOOR = float(np.log(1e-6))


def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p):
    p = np.asarray(p)
    return (p[O_W1:O_B1].reshape(NIN, NH), p[O_B1:O_W2], p[O_W2:O_B2].reshape(NH, NH), p[O_B2:O_W3],
            p[O_W3:O_B3], p[O_B3])


GELU_C0 = np.sqrt(2.0 / np.pi)
GELU_C1 = 0.044715


def gelu(x):
    """GELU in its tanh form (Hendrycks & Gimpel, 2016), as the kernels use it."""
    return 0.5 * x * (1.0 + np.tanh(GELU_C0 * (x + GELU_C1 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(GELU_C0 * (x + GELU_C1 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_C0 * (1.0 + 3.0 * GELU_C1 * x * x)


def forward(p, x, bf16_ops=True):
    """Network output y [n] for normalised features x [n, 8] (mlp.cu k_mlp_train forward)."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    if bf16_ops:
        xb = bf16(x).astype(np.float64)
        z1 = xb @ bf16(W1).astype(np.float64) + b1.astype(np.float64)
        h1 = bf16(gelu(z1).astype(np.float32)).astype(np.float64)
        z2 = h1 @ bf16(W2).astype(np.float64) + b2.astype(np.float64)
    else:
        z1 = x.astype(np.float64) @ W1.astype(np.float64) + b1
        h1 = gelu(z1)
        z2 = h1 @ W2.astype(np.float64) + b2
    y = gelu(z2) @ w3.astype(np.float64) + float(b3)
    return y


def grad(p, x, t, bf16_ops=True):
    """(gradient [NP], loss) of mean((y - t)^2) over the rows of x."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    n = x.shape[0]
    x64 = bf16(x).astype(np.float64) if bf16_ops else x.astype(np.float64)
    W1e = bf16(W1).astype(np.float64) if bf16_ops else W1.astype(np.float64)
    W2e = bf16(W2).astype(np.float64) if bf16_ops else W2.astype(np.float64)
    z1 = x64 @ W1e + b1
    h1 = gelu(z1)
    if bf16_ops:
        h1 = bf16(h1.astype(np.float32)).astype(np.float64)
    z2 = h1 @ W2e + b2
    h2 = gelu(z2)
    y = h2 @ w3.astype(np.float64) + float(b3)
    r = y - t.astype(np.float64)
    loss = float(np.mean(r * r))
    dy = 2.0 * r / n
    g2 = dy[:, None] * w3[None, :] * gelu_grad(z2)
    g2e = bf16(g2.astype(np.float32)).astype(np.float64) if bf16_ops else g2
    d1 = (g2e @ W2e.T) * gelu_grad(z1)
    # the weight gradients are a BF16 GEMM on the GPU (FP32 accumulation):
    # g2, delta1, h2 and dy enter it rounded to BF16; db3 is an FP32 sum
    rb = (lambda a: bf16(a.astype(np.float32)).astype(np.float64)) if bf16_ops else (lambda a: a)
    d1e, h2e, dye = rb(d1), rb(h2), rb(dy)
    g = np.zeros(NP)
    g[O_W3:O_B3] = h2e.T @ dye
    g[O_B3] = dy.sum()
    g[O_B2:O_W3] = g2e.sum(0)
    g[O_W2:O_B2] = (h1.T @ g2e).ravel()
    g[O_B1:O_W2] = d1e.sum(0)
    g[O_W1:O_B1] = (x64.T @ d1e).ravel()
    return g, loss


def raw_features(d, cs_prev, k, dz, delta, log_delta_z0, wall, dtdz=None, beta=0.0):
    """The 8 transformed features at level k (mlp.cu raw_features).

    ``d`` maps 'dudx' .. 'dwdz' to (nz+2, ny, nx) arrays, ``cs_prev`` is the
    coefficient before the update; returns [ny*nx, 8] in float32 arithmetic.
    Level 1 is the uvp node (w-node quantities averaged up), levels >= 2 are
    w nodes (uvp quantities averaged down).  Features: log1p |S|,
    log1p S:S, log1p Omega:Omega, signed log1p tr(S^3), log1p(z / Delta),
    log max(Cs^2_prev, 1e-6), signed log1p of the vortex stretching
    w_i S_ij w_j, log(Delta / z0) -- or, for a buoyant run (``dtdz`` the
    scalar's vertical gradient on w nodes, ``beta`` = g/theta_0), the signed
    log1p of the gradient Richardson number beta dtdz / (uz^2 + vz^2 + 1e-12).
    """
    f = {key: np.asarray(a, np.float32) for key, a in d.items()}
    h = np.float32(0.5)
    if k == 1:
        ux, uy, vx, vy = f["dudx"][1], f["dudy"][1], f["dvdx"][1], f["dvdy"][1]
        uz = f["dudz"][1] if wall else h * (f["dudz"][1] + f["dudz"][2])
        vz = f["dvdz"][1] if wall else h * (f["dvdz"][1] + f["dvdz"][2])
        wx = h * (f["dwdx"][1] + f["dwdx"][2])
        wy = h * (f["dwdy"][1] + f["dwdy"][2])
        wz = f["dwdz"][1]
    else:
        ux = h * (f["dudx"][k] + f["dudx"][k - 1])
        uy = h * (f["dudy"][k] + f["dudy"][k - 1])
        uz = f["dudz"][k]
        vx = h * (f["dvdx"][k] + f["dvdx"][k - 1])
        vy = h * (f["dvdy"][k] + f["dvdy"][k - 1])
        vz = f["dvdz"][k]
        wx, wy = f["dwdx"][k], f["dwdy"][k]
        wz = h * (f["dwdz"][k] + f["dwdz"][k - 1])
    s11, s22, s33 = ux, vy, wz
    s12, s13, s23 = h * (uy + vx), h * (uz + wx), h * (vz + wy)
    o12, o13, o23 = h * (uy - vx), h * (uz - wx), h * (vz - wy)
    ss = s11 * s11 + s22 * s22 + s33 * s33 + 2 * (s12 * s12 + s13 * s13 + s23 * s23)
    smag = np.sqrt(2 * ss)
    oo = 2 * (o12 * o12 + o13 * o13 + o23 * o23)
    r3 = (s11 ** 3 + s22 ** 3 + s33 ** 3 + 3 * (s12 * s12 * (s11 + s22) + s13 * s13 * (s11 + s33) +
                                                  s23 * s23 * (s22 + s33)) + 6 * s12 * s13 * s23)
    z = np.float32(0.5 * dz if k == 1 else (k - 1) * dz)
    out = np.empty(smag.shape + (8,), np.float32)
    out[..., 0] = np.log1p(smag)
    out[..., 1] = np.log1p(ss)
    out[..., 2] = np.log1p(oo)
    out[..., 3] = np.copysign(np.log1p(np.abs(r3)), r3)
    out[..., 4] = np.log1p(z / np.float32(delta))
    out[..., 5] = np.log(np.maximum(np.asarray(cs_prev, np.float32)[k], np.float32(1e-6)))
    w1, w2, w3 = -2 * o23, 2 * o13, -2 * o12
    vs = s11 * w1 * w1 + s22 * w2 * w2 + s33 * w3 * w3 + 2 * (s12 * w1 * w2 + s13 * w1 * w3 + s23 * w2 * w3)
    out[..., 6] = np.copysign(np.log1p(np.abs(vs)), vs)
    if dtdz is not None:
        ri = np.float32(beta) * np.asarray(dtdz, np.float32)[k] / (uz * uz + vz * vz + np.float32(1e-12))
        out[..., 7] = np.copysign(np.log1p(np.abs(ri)), ri)
    else:
        out[..., 7] = np.float32(log_delta_z0)
    return out.reshape(-1, 8)


def cs_from_output(y, stats, log_cs_prev):
    """Cs^2 from the normalised output (k_mlp_infer's epilogue): the output,
    clamped to the trained target range, is the change of log Cs^2 from the
    floored previous coefficient (feature 5, unnormalised); log Cs^2 is then
    clamped to the range of feature 5 seen in training."""
    y = np.clip(np.asarray(y, np.float64), stats[S_YMIN], stats[S_YMAX])
    lc = np.asarray(log_cs_prev, np.float64) + stats[S_YMU] + stats[S_YSD] * y
    lo = stats[S_MU + 5] + stats[S_SD + 5] * stats[S_MIN + 5]
    hi = stats[S_MU + 5] + stats[S_SD + 5] * stats[S_MAX + 5]
    lc = np.clip(lc, lo, hi)
    return np.clip(np.exp(lc), 1e-24, 1.0)


def in_range(xn, stats):
    """True where every normalised feature lies within the training range
    +- (0.25 sd + 5 % of the range), as k_mlp_infer tests it."""
    mn, mx = stats[S_MIN:S_MIN + 8], stats[S_MAX:S_MAX + 8]
    margin = 0.25 + 0.05 * (mx - mn)
    lo = mn - margin
    hi = mx + margin
    return np.all((xn >= lo) & (xn <= hi), axis=-1)
