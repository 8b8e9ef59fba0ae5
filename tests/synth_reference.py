"""Float64 torch restatement of the real-valued decode operator D (test infrastructure): the
reference's decode (Core/idx2Decode.cpp:141-320) with the integer inverse zfp (Core/Zfp.h:181)
replaced by its real form, written as explicit linear maps: the 4x4 matrix of one inverse zfp
line and the 33x33 matrix of one inverse CDF5/3 line (Core/Wavelet.h:250), both built from their
step definitions, the subband weights of GetCdf53NormsFast (Core/Wavelet.h:19), the low-band
hand-off from the parent brick (Core/idx2Decode.cpp:285-293). Autograd on it gives the FP64
reference gradient."""
import math

import numpy as np
import torch


def _rilift4(v):
    x, y, z, w = v
    y += w * 0.5
    w -= y * 0.5
    y += w
    w *= 2
    w -= y
    z += x
    x *= 2
    x -= z
    y += z
    z *= 2
    z -= y
    w += x
    x *= 2
    x -= w
    return [x, y, z, w]


def _rilift33(v):
    v = list(v)
    for x in range(1, 31, 2):
        V = v[x] * 0.25
        v[x - 1] -= V
        v[x + 1] -= V
    V = v[31] * 0.25
    v[30] -= V
    v[32] -= V
    for x in range(1, 31, 2):
        v[x] += (v[x - 1] + v[x + 1]) * 0.5
    v[31] += (v[32] + v[30]) * 0.5
    return v


def _matrix(f, n):
    m = np.zeros((n, n))
    for j in range(n):
        e = [0.0] * n
        e[j] = 1.0
        m[:, j] = f(e)
    return torch.tensor(m, dtype=torch.float64)


M4 = _matrix(_rilift4, 4)
K33 = _matrix(_rilift33, 33)


def _norms():
    scal, wave = [], []
    n1, n2 = 3.0, 23.0
    for i in range(16):
        scal.append(math.sqrt(n1 / (1 << (i + 1))))
        n1 = n1 * 4 - 1
        wave.append(math.sqrt(n2 / (1 << (i + 5))))
        n2 = n2 * 4 - 33
    return scal, wave


def level_bricks(dims, nlevels):
    is2d = dims[2] == 1
    nb = [math.ceil(dims[0] / 32), math.ceil(dims[1] / 32), 1 if is2d else math.ceil(dims[2] / 32)]
    out = [tuple(nb)]
    for _ in range(1, nlevels):
        nb = [math.ceil(nb[0] / 2), math.ceil(nb[1] / 2), 1 if is2d else math.ceil(nb[2] / 2)]
        out.append(tuple(nb))
    return out


def coeff_count(dims, nlevels):
    nbrick = 33 * 33 * (1 if dims[2] == 1 else 33)
    return sum(b[0] * b[1] * b[2] for b in level_bricks(dims, nlevels)) * nbrick


def _blocks_along(S, axis, M):
    """Apply the 4x4 map on the first 16 samples of `axis` (4 blocks); a 17th sample is a block
    of extent 1 on that axis and is left as it is."""
    n = S.shape[axis]
    head = S.narrow(axis, 0, 16)
    shp = list(head.shape)
    head = head.reshape(shp[:axis] + [4, 4] + shp[axis + 1:])
    head = torch.movedim(head, axis + 1, -1) @ M.T
    head = torch.movedim(head, -1, axis + 1).reshape(shp)
    if n == 16:
        return head
    return torch.cat([head, S.narrow(axis, 16, n - 16)], dim=axis)


def synth(c, dims, nlevels):
    """grid (nz, ny, nx) = D(c) for one field, c a float64 tensor of coeff_count elements."""
    is2d = dims[2] == 1
    nz = 1 if is2d else 33
    nbrick = 33 * 33 * nz
    scal, wave = _norms()
    lb = level_bricks(dims, nlevels)
    bases = [0]
    for b in lb:
        bases.append(bases[-1] + b[0] * b[1] * b[2] * nbrick)
    prev = None
    grid = None
    for l in range(nlevels - 1, -1, -1):
        bx, by, bz = lb[l]
        n = bx * by * bz
        C = c[bases[l]:bases[l + 1]].reshape(n, nz, 33, 33)
        F = torch.zeros(n, nz, 33, 33, dtype=c.dtype)
        coarsest = l == nlevels - 1
        subs = [(hx, hy, 0) for hx in (0, 1) for hy in (0, 1)] if is2d else \
            [(hx, hy, hz) for hx in (0, 1) for hy in (0, 1) for hz in (0, 1)]
        for hx, hy, hz in subs:
            S = C[:, hz::2, hy::2, hx::2] if not is2d else C[:, :, hy::2, hx::2]
            for axis in ((1, 2, 3) if not is2d else (2, 3)):
                S = _blocks_along(S, axis, M4)
            w = 1.0
            for h, active in ((hx, True), (hy, True), (hz, not is2d)):
                if active:
                    w *= wave[l] if h else scal[l]
            s0 = hx == 0 and hy == 0 and hz == 0
            if not (s0 and not coarsest):
                S = S / w
            if not is2d:
                F[:, hz::2, hy::2, hx::2] = S
            else:
                F[:, :, hy::2, hx::2] = S
        if not coarsest and not is2d:
            # the low band from the parent brick, on the positions of the full low-band blocks
            # that are coded there; in 2D every low-band block is coded on every level and
            # overwrites the parent's values (Core/idx2Decode.cpp:126-130, 285-293), so the
            # parent reaches nothing
            pbx, pby, pbz = lb[l + 1]
            for i in range(n):
                x, y, z = i % bx, (i // bx) % by, i // (bx * by)
                p = ((z // (1 if is2d else 2)) * pby + y // 2) * pbx + x // 2
                ox, oy, oz = (x % 2) * 16, (y % 2) * 16, (0 if is2d else (z % 2) * 16)
                if is2d:
                    F[i, 0, 0:32:2, 0:32:2] = prev[p, 0, oy:oy + 16, ox:ox + 16]
                else:
                    F[i, 0:32:2, 0:32:2, 0:32:2] = prev[p, oz:oz + 16, oy:oy + 16, ox:ox + 16]
        # inverse CDF5/3 along z, y, x
        if not is2d:
            F = torch.einsum("ij,njyx->niyx", K33, F)
        F = torch.einsum("ij,nzjx->nzix", K33, F)
        F = torch.einsum("ij,nzyj->nzyi", K33, F)
        if l > 0:
            prev = F
        else:
            grid = torch.zeros(dims[2], dims[1], dims[0], dtype=c.dtype)
            for i in range(n):
                x, y, z = i % bx, (i // bx) % by, i // (bx * by)
                gx, gy, gz = x * 32, y * 32, (z if is2d else z * 32)
                vx, vy, vz = min(32, dims[0] - gx), min(32, dims[1] - gy), (1 if is2d else min(32, dims[2] - gz))
                grid[gz:gz + vz, gy:gy + vy, gx:gx + vx] = F[i, :vz, :vy, :vx]
    return grid
