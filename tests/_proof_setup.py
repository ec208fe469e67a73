"""Synthetic proving keys and proof jobs for the proof-core and serving tests,
with the oracle computing the eleven commitments of one proof step by step."""
import ctypes

import numpy as np

from _loader import load
from oracle import oracle as O

mzk = load()


def delta(a, order):
    out = a.copy()
    for i in range(1, a.shape[0]):
        p = a[i - 1]
        out[i] = O.fr_op("sub", a[i], O.fr_op("add", p, p) if order == 2 else p)
        if order == 2 and i >= 2:
            out[i] = O.fr_op("add", out[i], a[i - 2])
    return out


class Setup:
    def __init__(self, ctx, k, seed, shared=None):
        """shared = (srs_host, srs_device_ptr, offsets): the key uses bases of
        a larger SRS buffer (offsets = g, lagrange, delta, double delta);
        otherwise it gets its own SRS of 4n bases laid out in that order."""
        self.ctx, self.k = ctx, k
        self.g = mzk.EvaluationDomain(ctx, 5, k)
        self.o = O.Domain(5, k)
        n, E = self.g.n, self.g.extended_len
        self.n, self.E = n, E
        rnd = iter(range(seed * 1000, seed * 1000 + 900))
        col = lambda m: O.rand_fr(next(rnd), m)
        self.fixed = [col(E) for _ in range(7)]
        self.sigma = [col(E) for _ in range(3)]
        self.l0, self.ll, self.la = col(E), col(E), col(E)
        self.keep = []
        if shared is None:
            self.srs = O.gen_bases(seed + 7, 4 * n)  # g | lagrange | delta | double delta
            srs_ptr, self.offs = None, (0, n, 2 * n, 3 * n)
        else:
            self.srs, srs_ptr, self.offs = shared
        dev = self.dev
        pk = mzk.ProvingKeyDesc()
        pk.k = k
        for i in range(7):
            pk.fixed_ext[i] = dev(self.fixed[i])
        for i in range(3):
            pk.sigma_ext[i] = dev(self.sigma[i])
        pk.l0_ext, pk.l_last_ext, pk.l_active_ext = dev(self.l0), dev(self.ll), dev(self.la)
        pk.srs, pk.srs_len = (dev(self.srs) if srs_ptr is None else srs_ptr), self.srs.shape[0]
        pk.off_g, pk.off_lagrange, pk.off_lagrange_delta, pk.off_lagrange_double_delta = self.offs
        pk.blinding_factors = 7
        # Lagrange forms for device-derived z / h / Z
        self.sigma_lag = [col(n) for _ in range(3)]
        self.table_lag, self.sel_lag = col(n), col(n)
        for i in range(3):
            pk.sigma_lagrange[i] = dev(self.sigma_lag[i])
        pk.table_lagrange, pk.selector_lagrange = dev(self.table_lag), dev(self.sel_lag)
        self.pk = pk
        self.rnd = rnd

    def dev(self, a):
        b = self.ctx.alloc(a.nbytes)
        b.upload(a)
        self.keep.append(b)
        return b.ptr

    def job(self, seed):
        n = self.n
        w = {name: O.rand_fr(seed * 50 + i, n) for i, name in enumerate(["a", "b", "c", "z", "m", "h", "Z"])}
        ch = {name: O.rand_fr(seed * 50 + 20 + i, 1)[0] for i, name in enumerate(["y", "beta", "gamma", "theta"])}
        blinds = O.rand_fr(seed * 50 + 30, 3)
        j = mzk.ProofJob()
        for i, name in enumerate("abc"):
            j.advice[i] = self.dev(w[name])
        j.perm_z, j.lookup_m, j.lookup_h, j.lookup_Z = self.dev(w["z"]), self.dev(w["m"]), self.dev(w["h"]), self.dev(w["Z"])
        for name in ("y", "beta", "gamma", "theta"):
            getattr(j, name)[:] = [int(v) for v in ch[name]]
        for i in range(3):
            j.quotient_blinds[i][:] = [int(v) for v in blinds[i]]
        return j, w, ch, blinds

    def oracle(self, w, ch, blinds):
        n, o = self.n, self.o
        g, lag, dl, ddl = (self.srs[o:o + n] for o in self.offs)
        coms = [O.msm_best(w["a"], lag), O.msm_best(w["b"], lag), O.msm_best(w["c"], lag),
                O.msm_best(delta(w["m"], 1), dl), O.msm_best(delta(w["z"], 1), dl),
                O.msm_best(delta(w["Z"], 2), ddl), O.msm_best(w["h"], lag)]
        ext = {name: o.coeff_to_extended(o.lagrange_to_coeff(w[name])) for name in w}
        cols = {
            "advice": [ext["a"], ext["b"], ext["c"]], "fixed": self.fixed, "gate_fixed": [0, 1, 2, 3, 4],
            "gate_advice": [0, 1, 2], "perm_cols": [(0, 0), (0, 1), (0, 2)], "perm_sigma": self.sigma,
            "perm_z": [ext["z"]], "chunk_len": 3, "blinding_factors": 7, "l0": self.l0, "l_last": self.ll,
            "l_active": self.la, "lookup": {"input": 0, "table": 5, "selector": 6, "h": ext["h"], "z": ext["Z"],
                                            "m": ext["m"]},
            "extended_omega": o.get(2), "g_coset": o.get(3), **ch,
        }
        hd = mzk.build_quotient_desc(cols, self.k, self.g.extended_k, lambda a: a.ctypes.data)
        od = O.QuotientDesc()
        ctypes.memmove(ctypes.byref(od), ctypes.byref(hd), ctypes.sizeof(od))
        h = o.extended_to_coeff(o.quotient_eval(od, True))
        for i in range(4):
            limb = np.concatenate([h[i * (n - 1):(i + 1) * (n - 1)],
                                   (blinds[i] if i < 3 else np.zeros(4, np.uint64)).reshape(1, 4)])
            if i > 0:
                limb[0] = O.fr_op("sub", limb[0], blinds[i - 1])
            coms.append(O.msm_best(limb, g))
        return coms
