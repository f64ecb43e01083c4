"""CPU oracle of the learned closure model (test infrastructure only).

Restates in numpy the model that nse2d-channel-gpu_b200/csrc/closure.cu runs on the tensor
cores: inputs (omega/s0, psi/s1, u/s2, v/s3, y) per point, four 3x3 convolutions
5 -> H -> H -> H -> 1 with GELU (tanh form) after the first three, periodic in x and
zero-padded beyond the walls, on pixel-major [Ny, Nx, C] activations; the loss is the mean
over the interior pixels of a batch of fields of (z - tau / tau_scale)^2. The reference has no
closure model, so there are no reference vectors for it; the oracle is pinned instead by
central finite differences of its own loss in float64 (tests/test_closure_oracle.py).

With bf=True the forward and backward passes round where the GPU path rounds: the scaled
inputs, the weights, the hidden activations after GELU, and dZ before the input-gradient
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


C_GELU = np.sqrt(2.0 / np.pi)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C_GELU * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(C_GELU * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C_GELU * (1.0 + 3 * 0.044715 * x * x)


def inputs(w, psi, u, v, y, scales):
    """[Ny, Nx, 5]: omega, psi, u, v over their scales, and y."""
    s0, s1, s2, s3 = scales[0]
    yy = np.broadcast_to(np.asarray(y, np.float64)[:, None], np.shape(w))
    return np.stack([w / s0, psi / s1, u / s2, v / s3, yy], axis=-1)


def forward(params, x, bf=False):
    """params: [(W [cout, 9, cin], b [cout])] * 4; x: the [Ny, Nx, 5] inputs.
    Returns the per-layer (input h, im2col A, pre-activation z)."""
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    h = r(x)
    cache = []
    for layer, (W, b) in enumerate(params):
        A = im2col(h)
        z = np.einsum("jitc,otc->jio", A, r(W)) + np.asarray(b, np.float64)
        cache.append((h, A, z))
        if layer < len(params) - 1:
            h = r(gelu(z))
    return cache


def predict(params, w, psi, u, v, y, scales, bf=False):
    """tau (zero on the wall rows) of one field."""
    z = forward(params, inputs(w, psi, u, v, y, scales), bf)[-1][2][:, :, 0] * scales[1]
    z[0] = z[-1] = 0.0
    return z


def loss_and_grads(params, samples, y, scales, bf=False):
    """Loss of a batch of samples [(w, psi, u, v, tau)] and the gradients [(dW, db)] of every layer."""
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    Ny, Nx = np.shape(samples[0][0])
    pint = len(samples) * Nx * (Ny - 2)
    loss = 0.0
    grads = [(np.zeros_like(np.asarray(W, np.float64)), np.zeros(len(b))) for W, b in params]
    for (w, psi, u, v, tau) in samples:
        cache = forward(params, inputs(w, psi, u, v, y, scales), bf)
        z = cache[-1][2][:, :, 0]
        d = np.zeros_like(z)
        d[1:-1] = z[1:-1] - np.asarray(tau)[1:-1] / scales[1]
        loss += float((d ** 2).sum() / pint)
        dz = (2.0 * d / pint)[:, :, None]
        for layer in range(len(params) - 1, -1, -1):
            h, A, zl = cache[layer]
            W = params[layer][0]
            gw, gb = grads[layer]
            grads[layer] = (gw + np.einsum("jio,jitc->otc", dz, A), gb + dz.sum(axis=(0, 1)))
            if layer == 0:
                break
            dA = np.einsum("jio,otc->jitc", r(dz), r(W))
            dz = col2im(dA) * gelu_grad(cache[layer - 1][2])
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
