"""CPU oracle of the Fourier neural operator surrogate (test infrastructure only).

A numpy restatement of the network of sdc_b200/csrc/fno.cu (no reference counterpart:
jceyy/sdc has no learned component): forward pass, mean-squared-error loss and its exact
gradient by hand-written reverse mode. With ``bf16=True`` it rounds to BF16 (nearest
even) at the points where the library stores BF16 values -- every GEMM operand and the
DFT matrices -- and accumulates in float64, so it differs from the library only by
accumulation order; with ``bf16=False`` everything is float64, which is what the
finite-difference check of the gradient uses.

Array layout as in the library: x, y [B][ny][nx][C]; parameter vector
P [W][C], p [W]; per layer W_l [W][W], b_l [W], R_l [2m][m][2][W][W]; Q1 [H][W], q1 [H];
Q2 [C][H], q2 [C].
"""
import math

import numpy as np

try:
    from scipy.special import erf as _erf
except ImportError:  # pragma: no cover
    _erf = np.vectorize(math.erf)


def round_bf16(x):
    """float -> nearest-even BF16 value (as float32), via the float32 bit pattern."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


class FNOOracle:
    def __init__(self, nx, ny, C, width, modes, layers, hidden, bf16=True):
        self.nx, self.ny, self.C, self.W, self.m, self.nl, self.H = nx, ny, C, width, modes, layers, hidden
        self.my = 2 * modes
        self.bf16 = bf16
        W, m, my, H = width, modes, self.my, hidden
        self.shapes = [("P", (W, C)), ("p", (W,))]
        for l in range(layers):
            self.shapes += [(f"W{l}", (W, W)), (f"b{l}", (W,)), (f"R{l}", (my, m, 2, W, W))]
        self.shapes += [("Q1", (H, W)), ("q1", (H,)), ("Q2", (C, H)), ("q2", (C,))]
        self.nparam = sum(int(np.prod(s)) for _, s in self.shapes)
        self._dft()

    def rb(self, x):
        return round_bf16(x).astype(np.float64) if self.bf16 else np.asarray(x, np.float64)

    def unpack(self, v):
        out, o = {}, 0
        for name, s in self.shapes:
            n = int(np.prod(s))
            out[name] = np.asarray(v[o:o + n], np.float64).reshape(s)
            o += n
        return out

    def pack(self, d):
        return np.concatenate([d[name].reshape(-1) for name, _ in self.shapes])

    def _dft(self):
        nx, ny, m, my = self.nx, self.ny, self.m, self.my
        kx = np.arange(m)[:, None]
        x = np.arange(nx)[None, :]
        a = 2 * np.pi * ((kx * x) % nx) / nx
        # the library rounds double -> float -> BF16; the unrounded oracle keeps float64
        q = (lambda v: self.rb(np.asarray(v, np.float64).astype(np.float32))) if self.bf16 else \
            (lambda v: np.asarray(v, np.float64))
        self.Fx = np.concatenate([q(np.cos(a)), q(-np.sin(a))], axis=0)                 # [2m][nx]
        w = np.where(np.arange(m) == 0, 1.0, 2.0)[:, None] / (nx * ny)
        self.Gx = np.concatenate([q(w * np.cos(a)), q(-w * np.sin(a))], axis=0).T       # [nx][2m]
        ki = np.arange(my)
        ky = np.where(ki < m, ki, ki - my)[:, None]
        y = np.arange(ny)[None, :]
        b = 2 * np.pi * (((ky * y) % ny + ny) % ny) / ny
        c, s = q(np.cos(b)), q(np.sin(b))                                                # [my][ny]
        Fy = np.zeros((my, 2, ny, 2))
        Fy[:, 0, :, 0], Fy[:, 0, :, 1], Fy[:, 1, :, 0], Fy[:, 1, :, 1] = c, s, -s, c
        Gy = np.zeros((ny, 2, my, 2))
        Gy[:, 0, :, 0], Gy[:, 0, :, 1], Gy[:, 1, :, 0], Gy[:, 1, :, 1] = c.T, -s.T, s.T, c.T
        self.Fy, self.Gy = Fy, Gy

    def spectral_conv(self, h, Rc):
        """K(h) of one spectral layer from the same DFT matrices, without rounding:
        h [B][ny][nx][W], Rc complex [2m][m][W][W] -> [B][ny][nx][W]."""
        B, ny, nx, W = h.shape
        m = self.m
        A1 = np.einsum("kx,byxc->bykc", self.Fx, h).reshape(B, ny, 2, m, W)
        Ah = np.einsum("aiyr,byrkc->baikc", self.Fy, A1)
        Yc = np.einsum("bakc,akco->bako", Ah[:, :, 0] + 1j * Ah[:, :, 1], Rc)
        Yh = np.stack([Yc.real, Yc.imag], axis=2)
        Z = np.einsum("yrai,baiko->byrko", self.Gy, Yh).reshape(B, ny, 2 * m, W)
        return np.einsum("xk,byko->byxo", self.Gx, Z)

    # ---------------------------------------------------------------- forward
    def forward(self, v, x):
        p = self.unpack(v)
        rb, m, W = self.rb, self.m, self.W
        B, ny, nx, C = x.shape
        cache = {"x0": rb(x)}
        h = rb(cache["x0"] @ rb(p["P"]).T + p["p"])
        hs, pres, ahats = [h], [], []
        for l in range(self.nl):
            A1 = rb(np.einsum("kx,byxc->bykc", self.Fx, h))                     # [B][y][2m][W]
            A1 = A1.reshape(B, ny, 2, m, W)
            Ah = rb(np.einsum("aiyr,byrkc->baikc", self.Fy, A1))                 # [B][my][2][m][W]
            R = rb(p[f"R{l}"])                                                   # [my][m][2][W][W]
            Xc = Ah[:, :, 0] + 1j * Ah[:, :, 1]                                  # [B][my][m][W]
            Rc = R[:, :, 0] + 1j * R[:, :, 1]
            Yc = np.einsum("bakc,akco->bako", Xc, Rc)
            Yh = np.stack([rb(Yc.real), rb(Yc.imag)], axis=2)                    # [B][my][2][m][W]
            Z = rb(np.einsum("yrai,baiko->byrko", self.Gy, Yh))                  # [B][ny][2][m][W]
            Kv = np.einsum("xk,byko->byxo", self.Gx, Z.reshape(B, ny, 2 * m, W))
            pre = h @ rb(p[f"W{l}"]).T + p[f"b{l}"] + Kv
            h = rb(gelu(pre)) if l + 1 < self.nl else rb(pre)
            pres.append(pre)
            ahats.append(Ah)
            hs.append(h)
        q1pre = h @ rb(p["Q1"]).T + p["q1"]
        q1 = rb(gelu(q1pre))
        out = q1 @ rb(p["Q2"]).T + p["q2"]
        cache.update(hs=hs, pres=pres, ahats=ahats, q1pre=q1pre, q1=q1)
        return out, cache

    # ---------------------------------------------------------------- backward
    def loss_grad(self, v, x, target):
        p = self.unpack(v)
        rb, m, W, nl = self.rb, self.m, self.W, self.nl
        out, c = self.forward(v, x)
        B, ny, nx, C = x.shape
        n = out.size
        d = out - target
        loss = float(np.mean(d * d))
        g = {}
        sum_rows = lambda a: a.reshape(-1, a.shape[-1])
        gout = rb(2.0 * d / n)
        g["Q2"] = sum_rows(gout).T @ sum_rows(c["q1"])
        g["q2"] = sum_rows(gout).sum(0)
        g1 = rb((gout @ rb(p["Q2"])) * gelu_grad(c["q1pre"]))
        g["Q1"] = sum_rows(g1).T @ sum_rows(c["hs"][nl])
        g["q1"] = sum_rows(g1).sum(0)
        gp = rb(g1 @ rb(p["Q1"]))
        for l in range(nl - 1, -1, -1):
            h = c["hs"][l]
            g[f"W{l}"] = sum_rows(gp).T @ sum_rows(h)
            g[f"b{l}"] = sum_rows(gp).sum(0)
            dZ = rb(np.einsum("xk,byxo->byko", self.Gx, gp)).reshape(B, ny, 2, m, W)
            dY = rb(np.einsum("yrai,byrko->baiko", self.Gy, dZ))                 # [B][my][2][m][W]
            R = rb(p[f"R{l}"])
            Ah = c["ahats"][l]
            gr, gi = dY[:, :, 0], dY[:, :, 1]                                    # [B][my][m][W]
            ar, ai = Ah[:, :, 0], Ah[:, :, 1]
            Rr, Ri = R[:, :, 0], R[:, :, 1]                                      # [my][m][W][W]
            dAr = np.einsum("bako,akio->baki", gr, Rr) + np.einsum("bako,akio->baki", gi, Ri)
            dAi = -np.einsum("bako,akio->baki", gr, Ri) + np.einsum("bako,akio->baki", gi, Rr)
            dRr = np.einsum("bako,baki->akio", gr, ar) + np.einsum("bako,baki->akio", gi, ai)
            dRi = -np.einsum("bako,baki->akio", gr, ai) + np.einsum("bako,baki->akio", gi, ar)
            g[f"R{l}"] = np.stack([dRr, dRi], axis=2)
            dAh = np.stack([rb(dAr), rb(dAi)], axis=2)                           # [B][my][2][m][W]
            dA1 = rb(np.einsum("aiyr,baikc->byrkc", self.Fy, dAh)).reshape(B, ny, 2 * m, W)
            dhs = np.einsum("kx,bykc->byxc", self.Fx, dA1)
            dh = gp @ rb(p[f"W{l}"]) + dhs
            gp = rb(dh * gelu_grad(c["pres"][l - 1])) if l > 0 else rb(dh)
        g["P"] = sum_rows(gp).T @ sum_rows(c["x0"])
        g["p"] = sum_rows(gp).sum(0)
        return loss, self.pack(g)
