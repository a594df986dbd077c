"""FP64 reference of the differentiable shading stage -- test infrastructure.

The same model as csrc/shade.cu, evaluated in float64 with numpy: a forward,
its analytic gradient, and central finite differences of the forward.  The
G-buffer it consumes is rebuilt here from the oracle's own visibility, shadow
and secondary outputs (gbuffer_from_oracle), so the GPU G-buffer is checked
too.  Model terms cite the reference shaders they restate:
  sun A*SUN*lit*max(n.s,0) and sky A*K*0.5 (resolve.wgsl:746-756,786-787),
  water under*tr + body*(1-tr) with tr = exp(-alpha*d) (common.wgsl:1262-1265),
  fog c*T + K*(1-T), T = exp(-clamp(rho * L, 0, 60)) with L the fog length
  e * path of transmittance_from (common.wgsl:1332-1341).
"""
from __future__ import annotations

import numpy as np

NP = 778
P_SUN, P_SKY, P_FOG, P_ABS = 768, 771, 774, 775
WATER = 13
G_HIT, G_LIT, G_TRACED, G_HIT2, G_FLIP = 1 << 11, 1 << 12, 1 << 13, 1 << 14, 1 << 15
G_SOFT, G_SOFT_SHIFT = 1 << 30, 27        # soft shadows: blocked rays of SOFT_SAMPLES in bits 27-29
SOFT_SAMPLES = 4
SPEC_SOFT_RAYS = 256                      # VM_SPEC_SOFT_RAYS: jittered rays, blocked fraction

NORMALS = np.array([[-1, 0, 0], [1, 0, 0], [0, -1, 0], [0, 1, 0], [0, 0, -1], [0, 0, 1],
                    [0.70710678, 0, -0.70710678], [0.70710678, 0, 0.70710678]], np.float64)


def fog_length(y0, s, rdy, falloff, height):
    """e * path of transmittance_from (common.wgsl:1332-1341), float64: the
    fog's optical length per unit density."""
    x = min(max(falloff * s * rdy, -60.0), 60.0)
    path = s * (1.0 - np.exp(-x)) / x if abs(x) > 1e-4 else s
    return float(np.exp(-min(max(falloff * (y0 - height), -60.0), 60.0)) * path)


def gbuffer_from_oracle(oracle, vis, shadow, sec_key, sec_t, fog_falloff, fog_height):
    """The G-buffer (vm_shade_gbuf) of one view from the oracle's outputs,
    with the fog length in float64 (the device's is float32)."""
    f = oracle.frame
    w, h = int(f.res[0]), int(f.res[1])
    n = w * h
    code = np.zeros(n, np.uint32)
    t = np.zeros(n, np.float32)
    d = np.zeros(n, np.float32)
    fog = np.zeros(n, np.float64)
    y0 = float(np.float32(f.cam_pos[1]))
    _, _, tt = oracle.expand(vis, (0, 0, 0), (1, 1, 1))
    for i in range(n):
        key = int(vis[i])
        if key == 0:
            continue
        px, py = i % w, i // w
        rd = oracle.ray_dir(px + 0.5, py + 0.5)
        low = key & 0xFFFFFF
        v = [(low >> 16) & 63, (low >> 8) & 63, low & 63]
        ci = (key >> 24) & 0x1FFF
        nid = (key >> 37) & 7
        bid = oracle.block_at(ci, v)
        c = (bid & 0xFF) | (nid << 8) | G_HIT | (G_LIT if shadow[i] == 0.0 else 0)
        if int(oracle.spec) & SPEC_SOFT_RAYS:
            c |= G_SOFT | (int(float(shadow[i]) * SOFT_SAMPLES + 0.5) << G_SOFT_SHIFT)
        nf = NORMALS[nid].astype(np.float32)
        if nid >= 6 and (nf[0] * rd[0] + nf[1] * rd[1]) + nf[2] * rd[2] > np.float32(0.0):
            c |= G_FLIP
        t[i] = tt[i]
        fog[i] = fog_length(y0, float(tt[i]), float(rd[1]), fog_falloff, fog_height)
        sk = int(sec_key[i])
        if bid == WATER and (sk >> 63):
            c |= G_TRACED
            d[i] = sec_t[i]
            if (sk >> 62) & 1:
                low2 = sk & 0xFFFFFF
                v2 = [(low2 >> 16) & 63, (low2 >> 8) & 63, low2 & 63]
                ci2 = (sk >> 24) & 0x1FFF
                bid2 = oracle.block_at(ci2, v2)
                c |= G_HIT2 | ((bid2 & 0xFF) << 16) | (((sk >> 37) & 7) << 24)
        code[i] = c
    g = np.zeros(n, dtype=[("code", "<u4"), ("t", "<f4"), ("d", "<f4"), ("fog", "<f8")])
    g["code"], g["t"], g["d"], g["fog"] = code, t, d, fog
    return g


class Model:
    """The shading model in float64 over a G-buffer (structured array)."""

    def __init__(self, g, sun_rgb):
        code = g["code"].astype(np.int64)
        self.hit = (code & G_HIT) != 0
        self.id = code & 0xFF
        self.nid = (code >> 8) & 7
        soft = (code & G_SOFT) != 0
        self.lit = np.where(soft, 1.0 - ((code >> G_SOFT_SHIFT) & 7) / SOFT_SAMPLES,
                            ((code & G_LIT) != 0).astype(np.float64))
        self.traced = (code & G_TRACED) != 0
        self.hit2 = (code & G_HIT2) != 0
        self.id2 = (code >> 16) & 0xFF
        self.nid2 = (code >> 24) & 7
        flip = (code & G_FLIP) != 0
        self.n = NORMALS[self.nid] * np.where(flip, -1.0, 1.0)[:, None]
        self.n2 = NORMALS[self.nid2]
        self.d = np.maximum(g["d"].astype(np.float64), 0.0)
        self.L = g["fog"].astype(np.float64)
        self.water = self.hit & (self.id == WATER)
        self.surf = self.hit & ~self.water
        self.S = np.asarray(sun_rgb, np.float64)

    def fog(self, rho):
        """T = exp(-clamp(rho * L, 0, 60)) and dT/drho."""
        tau = rho * self.L
        T = np.exp(-np.clip(tau, 0.0, 60.0))
        dT = np.where((tau > 0) & (tau < 60), -T * self.L, 0.0)
        return T, dT

    def _prefog(self, p):
        """The colour before fog, with the intermediates the gradient needs."""
        A = p[:768].reshape(256, 3)
        s = p[P_SUN:P_SUN + 3]
        sn = s / np.sqrt(s @ s)
        K = p[P_SKY:P_SKY + 3]
        alpha = p[P_ABS:P_ABS + 3]
        n = len(self.L)
        ndl = np.maximum(self.n @ sn, 0.0)
        ndl2 = np.maximum(self.n2 @ sn, 0.0)
        body = A[WATER] * K
        tr = np.exp(-alpha[None, :] * self.d[:, None])
        under = np.where(self.hit2[:, None], A[self.id2] * (self.S * ndl2[:, None] + 0.5 * K), 0.0)
        c = np.tile(K, (n, 1))
        surf, wt = self.surf, self.water
        c[surf] = A[self.id[surf]] * (self.S * (self.lit[surf] * ndl[surf])[:, None] + 0.5 * K)
        c[wt] = body
        trm = wt & self.traced
        c[trm] = (under * tr + body * (1 - tr))[trm]
        return c, dict(A=A, sn=sn, ls=np.sqrt(s @ s), K=K, ndl=ndl, ndl2=ndl2, body=body, tr=tr, under=under,
                       trm=trm)

    def forward(self, p):
        p = np.asarray(p, np.float64)
        c, m = self._prefog(p)
        K = m["K"]
        T, _ = self.fog(p[P_FOG])
        hit = self.hit
        c[hit] = c[hit] * T[hit][:, None] + K * (1 - T[hit])[:, None]
        return c

    def loss(self, p, target):
        e = self.forward(p) - np.asarray(target, np.float64)
        return float((e * e).sum())

    def grad(self, p, target):
        """Analytic dL/dp of the L2 loss, float64."""
        p = np.asarray(p, np.float64)
        c, m = self._prefog(p)
        A, sn, ls, K = m["A"], m["sn"], m["ls"], m["K"]
        ndl, ndl2, body, tr, under, trm = m["ndl"], m["ndl2"], m["body"], m["tr"], m["under"], m["trm"]
        T, dT = self.fog(p[P_FOG])
        hit = self.hit
        c_out = c.copy()
        c_out[hit] = c[hit] * T[hit][:, None] + K * (1 - T[hit])[:, None]
        dc_out = 2.0 * (c_out - np.asarray(target, np.float64))
        g = np.zeros(NP)
        gA = np.zeros((256, 3))
        gK = dc_out[~hit].sum(axis=0)
        gsn = np.zeros(3)
        # fog
        dTsum = (dc_out * (c - K)).sum(axis=1)
        g[P_FOG] = (dTsum * dT)[hit].sum()
        gK += (dc_out * (1 - T)[:, None])[hit].sum(axis=0)
        dc = dc_out * T[:, None]
        surf, wt = self.surf, self.water
        # surfaces
        shade = self.S * (self.lit * ndl)[:, None] + 0.5 * K
        np.add.at(gA, self.id[surf], (dc * shade)[surf])
        gK += (dc * A[self.id] * 0.5)[surf].sum(axis=0)
        dndl = (dc * A[self.id] * self.S).sum(axis=1) * self.lit
        msk = surf & (ndl > 0)
        gsn += (dndl[msk][:, None] * self.n[msk]).sum(axis=0)
        # water without a refraction leg
        wn = wt & ~self.traced
        gA[WATER] += (dc * K)[wn].sum(axis=0)
        gK += (dc * A[WATER])[wn].sum(axis=0)
        # water with a leg
        dunder = dc * tr
        dbody = dc * (1 - tr)
        dtr = dc * (under - body)
        g[P_ABS:P_ABS + 3] = (dtr * tr * (-self.d[:, None]))[trm].sum(axis=0)
        gA[WATER] += (dbody * K)[trm].sum(axis=0)
        gK += (dbody * A[WATER])[trm].sum(axis=0)
        h2 = trm & self.hit2
        np.add.at(gA, self.id2[h2], (dunder * (self.S * ndl2[:, None] + 0.5 * K))[h2])
        gK += (dunder * A[self.id2] * 0.5)[h2].sum(axis=0)
        dndl2 = (dunder * A[self.id2] * self.S).sum(axis=1)
        m2 = h2 & (ndl2 > 0)
        gsn += (dndl2[m2][:, None] * self.n2[m2]).sum(axis=0)
        g[:768] = gA.reshape(-1)
        g[P_SKY:P_SKY + 3] = gK
        g[P_SUN:P_SUN + 3] = (gsn - (gsn @ sn) * sn) / ls
        return g

    def grad_fd(self, p, target, idx, h=1e-4, richardson=False):
        """Central differences of the loss in float64 for parameters idx;
        with richardson, (4 D(h/2) - D(h)) / 3, which cancels the h^2 term
        (the fog density's loss is strongly curved: exp(-rho * L) with
        optical lengths of hundreds of voxels)."""
        p = np.asarray(p, np.float64)

        def central(i, hh):
            a, b = p.copy(), p.copy()
            a[i] += hh
            b[i] -= hh
            return (self.loss(a, target) - self.loss(b, target)) / (2 * hh)

        out = np.zeros(len(idx))
        for j, i in enumerate(idx):
            out[j] = (4 * central(i, h / 2) - central(i, h)) / 3 if richardson else central(i, h)
        return out
