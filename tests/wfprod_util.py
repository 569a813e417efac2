"""Small product cases shared by the CPU and GPU product tests."""
import numpy as np

from project1_b200 import inputs


def small_workload(**kw):
    base = dict(natom=2, lcut=3, nrad=2, lcutm=3, nradm=2, ngpt=100, ngptm=40, nk=2, nocc=3,
                nunocc=70, step_radius=2, vol=300.0, gaunt_density=0.3)
    base.update(kw)
    return inputs.WfprodWorkload("small", **base)


def shifted_pw(w, shift=(1, 0, 0), gshift=(0, 1, 0), drop=10):
    """A q != 0 style basis: the unoccupied list is a shifted, shorter sphere."""
    pw = inputs.pw_basis(w)
    pw["gpt2"] = np.ascontiguousarray(pw["gpt1"][: pw["gpt1"].shape[0] - drop] + np.array(shift, np.int32))
    pw["gshift"] = np.array(gshift, np.int32)
    return pw


def mt_numpy(mt, nk, nocc, nunocc, c1, c2):
    """wavefproducts2_mt with closed-form indices (lmstart(l,m) = nrad*(l^2 + l + m),
    ln1 = nrad*(l1 - |l-LL|)/2 + j): an independent restatement of the oracle's loops."""
    L, Lm, nr, nrm, na = mt["lcut"], mt["lcutm"], mt["nrad"], mt["nradm"], mt["natom"]
    g, integ, cexp = mt["gaunt"], mt["integral"], mt["cexp"]
    maxlm, maxllm = (L + 1) ** 2 * nr, (Lm + 1) ** 2 * nrm
    T = np.zeros((maxlm, maxllm, maxlm))
    for LL in range(Lm + 1):
        for MM in range(-LL, LL + 1):
            for l in range(L + 1):
                for m in range(-l, l + 1):
                    m1 = m + MM
                    for l1 in range(abs(l - LL), min(l + LL, L) + 1, 2):
                        gg = g[l1, l, LL, m + L, MM + Lm]
                        if gg == 0.0 or abs(m1) > l1:
                            continue
                        for nn in range(nrm):
                            I = nrm * (LL * LL + LL + MM) + nn
                            for j in range(nr):
                                o = nr * (l1 * l1 + l1 + m1) + j
                                ln1 = nr * ((l1 - abs(l - LL)) // 2) + j
                                for i in range(nr):
                                    T[o, I, nr * (l * l + l + m) + i] += integ[l * nr + i, ln1, LL * nrm + nn] * gg
    out = np.zeros((nk * nocc * nunocc, na * maxllm), complex)
    for k in range(nk):
        for a in range(na):
            mat = np.einsum("oIi,ni->noI", T, c1[k, :, a, :])           # (nocc, lm1, I)
            blk = np.einsum("po,noI->npI", c2[k, :, a, :], np.conj(mat))  # (nocc, nunocc, I)
            out[k * nocc * nunocc:(k + 1) * nocc * nunocc, a * maxllm:(a + 1) * maxllm] = \
                cexp[a] * blk.reshape(nocc * nunocc, maxllm)
    return out
