"""CPU oracle of the learned preconditioner network (test infrastructure only).

numpy restatement of the network the engine trains and applies (csrc/learned.cu):
4 periodic 3^3 convolutions, channels 2 -> 16 -> 16 -> 16 -> 1, ReLU after the
first three, input [r / rms(r), V / vscale] per state, output scaled back by
rms(r); loss sum_s |net_s - y_s / rms_s|^2 / sum_s |y_s / rms_s|^2 and its exact
gradient by hand-written backpropagation. Weights and stored activations are
rounded to bfloat16 as the device stores them; the arithmetic is FP64. The
reference has no preconditioner, so this checks the engine's own kernels
(forward and gradient) against an independent implementation.
"""
import numpy as np

CIN = (2, 16, 16, 16)
COUT = (16, 16, 16, 1)


def bf16(a):
    """Round to bfloat16 (nearest, ties to even) and return as float64."""
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params):
    """params (flat, per layer W[cout][cin][27] then b[cout]) -> [(W (cout,cin,3,3,3), b)]."""
    out, off = [], 0
    for ci, co in zip(CIN, COUT):
        w = np.asarray(params[off:off + co * ci * 27], dtype=np.float64).reshape(co, ci, 3, 3, 3)
        off += co * ci * 27
        b = np.asarray(params[off:off + co], dtype=np.float64)
        off += co
        out.append((w, b))
    return out


def n_params():
    return sum(co * ci * 27 + co for ci, co in zip(CIN, COUT))


def _shift(x, dz, dy, dx):
    # result[..., z, y, x] = x[..., z + dz, y + dy, x + dx] (periodic)
    return np.roll(x, shift=(-dz, -dy, -dx), axis=(-3, -2, -1))


def conv(x, w, b=None):
    """x (B, cin, nz, ny, nx), w (cout, cin, 3, 3, 3) indexed [dz][dy][dx] -> (B, cout, nz, ny, nx)."""
    B, ci = x.shape[:2]
    co = w.shape[0]
    out = np.zeros((B, co) + x.shape[2:])
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                xs = _shift(x, dz - 1, dy - 1, dx - 1)
                out += np.einsum("oc,bczyx->bozyx", w[:, :, dz, dy, dx], xs)
    if b is not None:
        out += b[None, :, None, None, None]
    return out


def conv_wgrad(x, d):
    """dW[o, c, dz, dy, dx] = sum_v d[b, o, v] x[b, c, v + off]."""
    co, ci = d.shape[1], x.shape[1]
    g = np.zeros((co, ci, 3, 3, 3))
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                xs = _shift(x, dz - 1, dy - 1, dx - 1)
                g[:, :, dz, dy, dx] = np.einsum("bozyx,bczyx->oc", d, xs)
    return g


def conv_dgrad(d, w):
    """dx[b, c, u] = sum_o sum_tap w[o, c, tap] d[b, o, u - off(tap)]."""
    B = d.shape[0]
    ci = w.shape[1]
    out = np.zeros((B, ci) + d.shape[2:])
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                ds = _shift(d, -(dz - 1), -(dy - 1), -(dx - 1))
                out += np.einsum("oc,bozyx->bczyx", w[:, :, dz, dy, dx], ds)
    return out


def _id(a):
    return np.asarray(a, dtype=np.float64)


def _inputs(grid, R, V, vscale, rnd=bf16):
    nx, ny, nz = grid
    R = np.asarray(R, dtype=np.float64)
    rms = np.sqrt(np.mean(R * R, axis=1))
    rms = np.where(rms > 0, rms, 1.0)
    B = R.shape[0]
    x0 = np.zeros((B, 2, nz, ny, nx))
    x0[:, 0] = rnd(R / rms[:, None]).reshape(B, nz, ny, nx)
    x0[:, 1] = rnd(np.asarray(V) / vscale).reshape(nz, ny, nx)[None]
    return x0, rms


def forward(params, grid, R, V, vscale, exact=False):
    """(acts, p, rms): activations per layer (bf16-rounded unless exact) and the output."""
    rnd = _id if exact else bf16
    layers = unpack(rnd(np.asarray(params, dtype=np.float64 if exact else np.float32)))
    biases = [np.asarray(b, dtype=np.float64) for _, b in unpack(params)]
    x, rms = _inputs(grid, R, V, vscale, rnd)
    acts = [x]
    for li, ((w, _), b) in enumerate(zip(layers, biases)):
        y = conv(acts[-1], w, b)
        if li < 3:
            acts.append(rnd(np.maximum(y, 0.0)))
        else:
            p = y[:, 0]
    return acts, p, rms


def apply(params, grid, R, V, vscale):
    """NN(R) in the units of R, (ns, N)."""
    _, p, rms = forward(params, grid, R, V, vscale)
    return p.reshape(p.shape[0], -1) * rms[:, None]


def loss_and_grad(params, grid, R, V, vscale, Y, exact=False):
    rnd = _id if exact else bf16
    layers = unpack(rnd(np.asarray(params, dtype=np.float64 if exact else np.float32)))
    acts, p, rms = forward(params, grid, R, V, vscale, exact)
    B = p.shape[0]
    t = (np.asarray(Y, dtype=np.float64) / rms[:, None]).reshape(p.shape)
    diff = p - t
    tn = np.sum(t * t)
    loss = np.sum(diff * diff) / tn
    d = (2.0 * diff / tn)[:, None]  # (B, 1, ...)
    grads = [None] * 4
    for li in range(3, -1, -1):
        w = layers[li][0]
        gw = conv_wgrad(acts[li], d)
        gb = d.sum(axis=(0, 2, 3, 4))
        grads[li] = (gw, gb)
        if li > 0:
            d = conv_dgrad(d, w) * (acts[li] > 0)
    flat = np.concatenate([np.concatenate([gw.reshape(-1), gb]) for gw, gb in grads])
    return loss, flat
