"""CPU oracle of the multigrid preconditioner (test infrastructure only).

Float64 numpy restatement of the horizontal aggregation multigrid V-cycle in
pincflow.jl_b200/csrc/pcf_mg.cuh and the mg_* functions of pcf_solver.cu,
used to check the GPU's hierarchy, coarse operators and V-cycle.  The
multigrid has no counterpart in the reference; its smoother is the
reference's pseudo-time line relaxation (apply_preconditioner!.jl:53-121,
restated here as in or_solver.cpp's precond_impl, with the Thomas pivots of
k_factors).

Operator arrays are (25, nz, ny, nx) in the reference Tensor order; vectors
(nz, ny, nx); x and y periodic, zero outside the z walls.
"""
from __future__ import annotations

import numpy as np

# (dx, dy, dz) of each plane in Tensor order (Tensor.jl:70-102, apply_operator!.jl:157-269)
OFFSETS = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1),
           (-1, 0, -1), (-1, 0, 1), (1, 0, -1), (1, 0, 1), (0, -1, -1), (0, -1, 1), (0, 1, -1), (0, 1, 1),
           (0, 0, -2), (0, 0, 2), (-1, 0, -2), (-1, 0, 2), (1, 0, -2), (1, 0, 2), (0, -1, -2), (0, -1, 2),
           (0, 1, -2), (0, 1, 2)]
INDEX = {o: p for p, o in enumerate(OFFSETS)}
AC, AD, AU = 0, 5, 6
HORIZONTAL = [p for p in range(25) if p not in (AC, AD, AU)]


def shift(s, off):
    """s at (i+dx, j+dy, k+dz): periodic in x, y; zero beyond the z walls."""
    dx, dy, dz = off
    t = np.roll(np.roll(s, -dx, axis=-1), -dy, axis=-2)
    if dz == 0:
        return t
    out = np.zeros_like(t)
    if dz > 0:
        out[:-dz] = t[dz:]
    else:
        out[-dz:] = t[:dz]
    return out


def apply(coef, s, planes=range(25)):
    out = np.zeros_like(s)
    for p in planes:
        out += coef[p] * shift(s, OFFSETS[p])
    return out


def bf16(a):
    """BF16 rounding (to nearest, ties to even) of the FP32 rounding of a, as
    the GPU's BF16 operator copies store it; returned as float64."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def e4m3(a):
    """Rounding to FP8 E4M3 (to nearest, ties to even; saturating at 448;
    subnormal step 2^-9), as cvt.rn.satfinite.e4m3x2.f32 does; float64 out."""
    a = np.asarray(a, dtype=np.float64)
    m = np.minimum(np.abs(a), 448.0)
    _, e = np.frexp(m)                      # m = f 2^e, f in [0.5, 1)
    e = np.maximum(e - 1, -6)               # the binade's exponent; subnormals share 2^-6's step
    q = np.ldexp(1.0, e - 3)                # 3 mantissa bits
    return np.sign(a) * np.minimum(np.round(m / q) * q, 448.0)


def fp8_planes(planes):
    """The GPU's FP8 copy of BF16-rounded planes, widened back: plane p as
    E4M3(c scale_p) / scale_p with scale_p = 2^(7 - e_p), max |c| = f 2^e_p."""
    out = np.zeros_like(planes)
    for p in range(planes.shape[0]):
        mx = np.abs(planes[p]).max()
        if mx == 0:
            continue
        _, e = np.frexp(np.float32(mx))
        sc = np.ldexp(1.0, 7 - int(e))
        out[p] = e4m3(planes[p] * sc) / sc
    return out


def factors(coef, deta):
    """Thomas pivots P, M, Q (k_factors)."""
    ac, ad, au = coef[AC], coef[AD], coef[AU]
    nz = ac.shape[0]
    P, M, Q = np.zeros_like(ac), np.zeros_like(ac), np.zeros_like(ac)
    q = np.zeros_like(ac[0])
    for k in range(nz):
        piv = 1 / (1 - deta * ac[k]) if k == 0 else 1 / (1 - deta * ac[k] - deta * ad[k] * q)
        P[k] = piv
        M[k] = 0 if k == 0 else deta * ad[k] * piv
        q = deta * au[k] * piv
        Q[k] = q
    return P, M, Q


def thomas(fac, rhs):
    P, M, Q = fac
    nz = rhs.shape[0]
    y = np.zeros_like(rhs)
    prev = np.zeros_like(rhs[0])
    for k in range(nz):
        prev = rhs[k] * P[k] + M[k] * prev
        y[k] = prev
    for k in range(nz - 2, -1, -1):
        y[k] = y[k] + Q[k] * y[k + 1]
    return y


def pseudo_step(coef, fac, deta, b, s):
    """One pseudo-time step of apply_preconditioner!.jl:53-121 from s (None: s = 0)."""
    t = -deta * b if s is None else s + deta * (apply(coef, s, HORIZONTAL) - b)
    return thomas(fac, t)


def level_dims(nx, ny, nz, min_columns):
    """[(nx, ny, nz, cx, cy)] finest first (cx, cy: aggregation from the finer level)."""
    out = [(nx, ny, nz, 1, 1)]
    while True:
        fx, fy, _, _, _ = out[-1]
        cx = 2 if fx % 2 == 0 and fx >= 4 else 1
        cy = 2 if fy % 2 == 0 and fy >= 4 else 1
        if cx * cy == 1 or fx * fy <= min_columns:
            return out
        out.append((fx // cx, fy // cy, nz, cx, cy))


def coarsen(coef, fc, cx, cy):
    """Level l+1 operator and fcscal from level l (k_mg_fc, k_mg_coarsen)."""
    nz, ny, nx = fc.shape
    NX, NY = nx // cx, ny // cy
    fcc = np.sqrt((fc ** 2).reshape(nz, NY, cy, NX, cx).mean(axis=(2, 4)))
    acc = np.zeros((25, nz, NY, NX))
    ia, jb = np.arange(nx) % cx, np.arange(ny) % cy
    for p, (dx, dy, dz) in enumerate(OFFSETS):
        a0 = fc * coef[p] * shift(fc, (dx, dy, dz))  # zero where k+dz is outside
        ox = np.floor_divide(ia + dx, cx) if cx == 2 else np.full(nx, dx)
        oy = np.floor_divide(jb + dy, cy) if cy == 2 else np.full(ny, dy)
        for vx in (-1, 0, 1):
            for vy in (-1, 0, 1):
                m = (oy == vy)[:, None] & (ox == vx)[None, :]
                if not m.any():
                    continue
                agg = (a0 * m).reshape(nz, NY, cy, NX, cx).sum(axis=(2, 4))
                acc[INDEX[(vx, vy, dz)]] += agg
    for p in HORIZONTAL:
        dx, dy, dz = OFFSETS[p]
        if dx == 0 and dy == 0:
            continue
        keep = 1.0 / cx if dx != 0 else 1.0 / cy
        moved = (1 - keep) * acc[p]
        acc[p] -= moved
        acc[INDEX[(0, 0, dz)]] += moved
    out = np.zeros_like(acc)
    for p, o in enumerate(OFFSETS):
        den = cx * cy * fcc * shift(fcc, o)
        out[p] = np.where(den > 0, acc[p] / np.where(den > 0, den, 1.0), 0.0)
    return out, fcc


class Multigrid:
    """The hierarchy and V-cycle of the GPU preconditioner (mg_prepare, mg_precond, mg_cycle)."""

    def __init__(self, coef, fcscal, dx, dy, dtau=1.0, coarse_iterations=4, min_columns=16, bf16_planes=False,
                 fp8_smoother=False):
        """bf16_planes: the residual and pseudo-step stencils of level 0, and
        of level 1 unless it is the coarsest, read BF16-rounded planes (the
        GPU's mg_operator_bf16); the Thomas pivots keep the unrounded operator.
        fp8_smoother (with bf16_planes): level 0's pseudo-time steps read the
        FP8 copy of those planes (the GPU's mg_smoother_fp8)."""
        nz, ny, nx = fcscal.shape
        self.dims = level_dims(nx, ny, nz, min_columns)
        self.ci = coarse_iterations
        self.levels = []
        ddx, ddy = dx, dy
        c, f = np.asarray(coef, dtype=np.float64), np.asarray(fcscal, dtype=np.float64)
        for l, (_, _, _, cx, cy) in enumerate(self.dims):
            if l > 0:
                c, f = coarsen(c, f, cx, cy)
                ddx, ddy = ddx * cx, ddy * cy
            deta = dtau / (2 * (1 / ddx ** 2 + 1 / ddy ** 2))
            self.levels.append(dict(coef=c, fc=f, deta=deta, fac=factors(c, deta), cx=cx, cy=cy))
        for l, L in enumerate(self.levels):
            rounded = bf16_planes and (l == 0 or (l == 1 and l < len(self.levels) - 1))
            L["scoef"] = bf16(L["coef"]) if rounded else L["coef"]
            L["pcoef"] = fp8_planes(L["scoef"]) if (fp8_smoother and bf16_planes and l == 0) else L["scoef"]

    def smooth(self, l, b, steps):
        L = self.levels[l]
        s = pseudo_step(L["pcoef"], L["fac"], L["deta"], b, None)
        for _ in range(steps - 1):
            s = pseudo_step(L["pcoef"], L["fac"], L["deta"], b, s)
        return s

    def cycle(self, b, l=0):
        L = self.levels[l]
        if l == len(self.levels) - 1:
            return self.smooth(l, b, self.ci)
        s = self.smooth(l, b, 1)
        r = b - apply(L["scoef"], s)
        C = self.levels[l + 1]
        cx, cy = C["cx"], C["cy"]
        nz, ny, nx = b.shape
        bc = (L["fc"] * r).reshape(nz, ny // cy, cy, nx // cx, cx).sum(axis=(2, 4)) / (cx * cy * C["fc"])
        e = self.cycle(bc, l + 1)
        s = s + np.repeat(np.repeat(C["fc"] * e, cy, axis=1), cx, axis=2) / L["fc"]
        return pseudo_step(L["pcoef"], L["fac"], L["deta"], b, s)


def bicgstab(coef, M, b, tol=1e-10, maxit=1000):
    """Flexible right-preconditioned BiCGSTAB (x accumulated from M p, M s), x0 = 0;
    returns (x, iterations, relative recursive residual)."""
    x = np.zeros_like(b)
    r = b.copy()
    r0 = r.copy()
    p = r.copy()
    bn = np.sqrt(np.mean(b * b))
    rho = np.vdot(r0, r)
    res = 1.0
    for it in range(1, maxit + 1):
        zp = M(p)
        v = apply(coef, zp)
        alpha = rho / np.vdot(r0, v)
        s = r - alpha * v
        zs = M(s)
        t = apply(coef, zs)
        omega = np.vdot(t, s) / np.vdot(t, t)
        x += alpha * zp + omega * zs
        r = s - omega * t
        res = np.sqrt(np.mean(r * r)) / bn
        if res <= tol:
            return x, it, res
        rn = np.vdot(r0, r)
        beta = rn / rho * alpha / omega
        rho = rn
        p = r + beta * (p - omega * v)
    return x, maxit, res
