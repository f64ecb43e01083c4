"""CPU oracle of the learned closure model (test infrastructure only).

Restates in numpy the model that nse2d-channel-gpu_b200/csrc/closure.cu runs on the tensor
cores: three 3x3 convolutions 2 -> H -> H -> 1 with ReLU after the first two, periodic in x and
zero-padded beyond the walls, on pixel-major [Ny, Nx, C] activations; the loss is the mean
over interior pixels of (z - tau / tau_scale)^2. The reference has no closure model, so there
are no reference vectors for it; the oracle is pinned instead by central finite differences
of its own loss in float64 (tests/test_closure_oracle.py).

With bf16=True the forward and backward passes round where the GPU path rounds: the scaled
inputs, the weights, the hidden activations after ReLU, and dZ before the input-gradient
product (round to nearest even, as __float2bfloat16_rn). Sums are float64 here and float32 on
the GPU.
"""
import numpy as np

TAPS = [(dy, dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]     # tap = 3 (dy + 1) + dx + 1


def bf16(x):
    """Round float values to bfloat16 (nearest even) and back to float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def im2col(h):
    """[Ny, Nx, C] -> [Ny, Nx, 9, C]: neighbour (j + dy, (i + dx) mod Nx), zero beyond the walls."""
    Ny, Nx, C = h.shape
    out = np.zeros((Ny, Nx, 9, C))
    for t, (dy, dx) in enumerate(TAPS):
        src = np.roll(h, -dx, axis=1)                 # src[:, i] = h[:, i + dx]
        if dy == 0:
            out[:, :, t, :] = src
        elif dy > 0:
            out[:-dy, :, t, :] = src[dy:]
        else:
            out[-dy:, :, t, :] = src[:dy]
    return out


def col2im(g):
    """Adjoint of im2col: [Ny, Nx, 9, C] -> [Ny, Nx, C]."""
    Ny, Nx, _, C = g.shape
    out = np.zeros((Ny, Nx, C))
    for t, (dy, dx) in enumerate(TAPS):
        part = np.zeros((Ny, Nx, C))
        if dy == 0:
            part[:] = g[:, :, t, :]
        elif dy > 0:
            part[dy:] = g[:-dy, :, t, :]
        else:
            part[:dy] = g[-dy:, :, t, :]
        out += np.roll(part, dx, axis=1)
    return out


def forward(params, w, psi, scales, bf=False):
    """params: [(W [cout, 9, cin], b [cout])] * 3; w, psi [Ny, Nx]; scales (sw, sp, st).
    Returns the per-layer (input h, im2col A, pre-activation z)."""
    r = bf16 if bf else (lambda x: np.asarray(x, dtype=np.float64))
    sw, sp, _ = scales
    h = r(np.stack([w / sw, psi / sp], axis=-1))
    cache = []
    for layer, (W, b) in enumerate(params):
        A = im2col(h)
        z = np.einsum("jitc,otc->jio", A, r(W)) + np.asarray(b, np.float64)
        cache.append((h, A, z))
        if layer < len(params) - 1:
            h = r(np.maximum(z, 0.0))
    return cache


def loss_and_grads(params, w, psi, tau, scales, bf=False):
    """Loss and the gradients [(dW, db)] of every layer."""
    r = bf16 if bf else (lambda x: np.asarray(x, dtype=np.float64))
    cache = forward(params, w, psi, scales, bf)
    z = cache[-1][2][:, :, 0]
    Ny, Nx = z.shape
    d = np.zeros_like(z)
    d[1:-1] = z[1:-1] - tau[1:-1] / scales[2]
    pint = Nx * (Ny - 2)
    loss = float((d ** 2).sum() / pint)
    dz = (2.0 * d / pint)[:, :, None]
    grads = [None] * len(params)
    for layer in range(len(params) - 1, -1, -1):
        h, A, zl = cache[layer]
        W = params[layer][0]
        grads[layer] = (np.einsum("jio,jitc->otc", dz, A), dz.sum(axis=(0, 1)))
        if layer == 0:
            break
        dA = np.einsum("jio,otc->jitc", r(dz), r(W))
        dh = col2im(dA)
        dz = dh * (cache[layer - 1][2] > 0)
    return loss, grads


def subgrid_target(J_fine_filtered, J_coarse):
    """tau = filter(J) - J(filter psi, filter omega), zero on the wall rows."""
    t = np.asarray(J_fine_filtered, np.float64) - np.asarray(J_coarse, np.float64)
    t[0] = 0.0
    t[-1] = 0.0
    return t


def box_filter(f, Nxc, Nyc):
    """CPU restatement of nse2d_box_filter."""
    Nyf, Nxf = f.shape
    rx, ry = Nxf // Nxc, (Nyf - 1) // (Nyc - 1)
    hx, hy = rx // 2, ry // 2
    out = np.zeros((Nyc, Nxc))
    for j in range(Nyc):
        for i in range(Nxc):
            s = ws = 0.0
            for e in range(-hy, hy + 1):
                jf = ry * j + e
                if jf < 0 or jf >= Nyf:
                    continue
                we = 0.5 if hy > 0 and abs(e) == hy else 1.0
                for dd in range(-hx, hx + 1):
                    wd = 0.5 if hx > 0 and abs(dd) == hx else 1.0
                    s += we * wd * f[jf, (rx * i + dd) % Nxf]
                    ws += we * wd
            out[j, i] = s / ws
    return out
