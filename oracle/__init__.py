"""CPU oracle for the SPEX polarisation hot path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, and only as the checker or the timed CPU baseline; the product never
imports it.

PARITY UNPINNED: the reference (SPEX 05.10, Fortran) cannot be compiled in this
image and ships no tests, golden vectors or fixtures for the path. The C
restatement (chi0_oracle.c, wfprod_oracle.c) follows the reference loops
line by line (citations in the C sources) and is cross-checked against an
independent numpy formulation (tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        srcs = list(HERE.glob("*.c")) + [HERE / "Makefile"]
        if not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in srcs):
            build()
        lib = C.CDLL(str(LIB))
        P, I64, I32, D = C.c_void_p, C.c_int64, C.c_int32, C.c_double
        lib.oracle_weights.argtypes = [I64, P, P, D, I32, P, P]
        lib.oracle_chi0_faithful.argtypes = [I64, I32, P, I64, P, I32, P, C.c_int]
        lib.oracle_chi0_accurate.argtypes = [I64, I32, P, I64, P, I32, P, C.c_int]
        lib.oracle_chi0_element.argtypes = [I64, P, P, P, I32, P]
        lib.oracle_scale.argtypes = [P, I64, D]
        lib.oracle_max_threads.restype = C.c_int
        lib.oracle_gen_cmatrix.argtypes = [C.c_uint64, C.c_uint32, I64, I64, I64, I64, D, P, C.c_int]
        lib.oracle_series_log.argtypes = [I64, P, P]
        lib.oracle_series_sincos_turns.argtypes = [I64, P, P, P]
        for name in ("oracle_weights", "oracle_chi0_faithful", "oracle_chi0_accurate",
                     "oracle_chi0_element", "oracle_scale", "oracle_gen_cmatrix",
                     "oracle_series_log", "oracle_series_sincos_turns"):
            getattr(lib, name).restype = None
        _lib = lib
    return _lib


def _p(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def gen_cmatrix(seed: int, stream_id: int, rows: int, cols: int, col0: int = 0,
                scale: float = 1.0, threads: int = 0) -> np.ndarray:
    """Columns [col0, col0+cols) of the seeded (rows x ...) complex stream matrix, as a
    Fortran (rows, cols) complex128 array: the projections the GPU library generates,
    bit for bit, without loading the library (inputs_oracle.c)."""
    out = np.empty((rows, cols), dtype=np.complex128, order="F")
    load().oracle_gen_cmatrix(seed, stream_id, rows, cols, rows, col0, scale, _p(out), threads)
    return out


def series_log(x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    load().oracle_series_log(x.size, _p(x), _p(y))
    return y


def series_sincos_turns(u):
    u = np.ascontiguousarray(u, dtype=np.float64)
    s, c = np.empty_like(u), np.empty_like(u)
    load().oracle_series_sincos_turns(u.size, _p(u), _p(s), _p(c))
    return s, c


def weights(ediff, omega, wscale=None, scale_all: float = 1.0) -> np.ndarray:
    """w (npair, nw), Fortran order (src/susceptibility.f:950-975)."""
    ediff = np.ascontiguousarray(ediff, dtype=np.float64)
    omega = np.ascontiguousarray(omega, dtype=np.float64)
    ws = None if wscale is None else np.ascontiguousarray(wscale, dtype=np.float64)
    w = np.zeros((ediff.shape[0], omega.shape[0]), dtype=np.float64, order="F")
    load().oracle_weights(ediff.shape[0], _p(ediff), _p(ws), scale_all, omega.shape[0], _p(omega), _p(w))
    return w


def chi0(cprod, w, accurate: bool = False, threads: int = 0, susceph=None) -> np.ndarray:
    """susceph (npack, nw) += body loop of src/susceptibility.f:1182-1240."""
    cprod = np.asfortranarray(cprod, dtype=np.complex128)
    w = np.asfortranarray(w, dtype=np.float64)
    npair, nbas = cprod.shape
    nw = w.shape[1]
    if susceph is None:
        susceph = np.zeros((nbas * (nbas + 1) // 2, nw), dtype=np.complex128, order="F")
    fn = load().oracle_chi0_accurate if accurate else load().oracle_chi0_faithful
    fn(npair, nbas, _p(cprod), npair, _p(w), nw, _p(susceph), threads)
    return susceph


def chi0_element(a, b, w) -> np.ndarray:
    """chi(i, j, :) for columns a = cprod(:, i), b = cprod(:, j); extended precision."""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    w = np.asfortranarray(w, dtype=np.float64)
    out = np.zeros(w.shape[1], dtype=np.complex128)
    load().oracle_chi0_element(a.shape[0], _p(a), _p(b), _p(w), w.shape[1], _p(out))
    return out


def max_threads() -> int:
    return load().oracle_max_threads()


def _bind_wfprod(lib):
    P, I64, D = C.c_void_p, C.c_int64, C.c_double
    ci = C.c_int
    lib.oracle_wfprod_mt.argtypes = [ci, ci, ci, ci, ci, P, P, ci, P, ci, ci, ci, P, P, P, I64]
    lib.oracle_wfprod_mt.restype = None
    lib.oracle_wfprod_pw.argtypes = [ci, P, ci, P, ci, P, P, ci, P, D, ci, ci, ci, P, P, P, I64, ci]
    lib.oracle_wfprod_pw.restype = None


def wfprod_mt(mt, nk, nocc, nunocc, cmt_occ, cmt_unocc, cprod, ldc=None):
    """cprod(:, :nbasp) += wavefproducts2_mt (src/wavefproducts.f:95-431). `mt` is the
    dict of project1_b200.inputs.mt_basis; cprod is Fortran (npair, nbas) complex."""
    lib = load()
    _bind_wfprod(lib)
    g = np.asfortranarray(mt["gaunt"], dtype=np.float64)
    integ = np.asfortranarray(mt["integral"], dtype=np.float64)
    ce = np.ascontiguousarray(mt["cexp"], dtype=np.complex128)
    c1 = np.ascontiguousarray(cmt_occ, dtype=np.complex128)
    c2 = np.ascontiguousarray(cmt_unocc, dtype=np.complex128)
    lib.oracle_wfprod_mt(mt["natom"], mt["lcut"], mt["nrad"], mt["lcutm"], mt["nradm"], _p(g), _p(integ),
                         integ.shape[1], _p(ce), nk, nocc, nunocc, _p(c1), _p(c2), _p(cprod),
                         cprod.shape[0] if ldc is None else ldc)
    return cprod


def wfprod_pw(pw, nk, nocc, nunocc, cpw_occ, cpw_unocc, cprod, col0, ldc=None):
    """cprod(:, col0:col0+ngptm) += explicit-convolution wavefproducts2_pw with the step
    function (src/wavefproducts.f:760-997)."""
    lib = load()
    _bind_wfprod(lib)
    gpt1 = np.ascontiguousarray(pw["gpt1"], dtype=np.int32)
    gpt2 = np.ascontiguousarray(pw["gpt2"], dtype=np.int32)
    gptm = np.ascontiguousarray(pw["gptm"], dtype=np.int32)
    gsh = np.ascontiguousarray(pw["gshift"], dtype=np.int32)
    cs = np.ascontiguousarray(pw["cstep"], dtype=np.complex128)
    c1 = np.ascontiguousarray(cpw_occ, dtype=np.complex128)
    c2 = np.ascontiguousarray(cpw_unocc, dtype=np.complex128)
    lib.oracle_wfprod_pw(gpt1.shape[0], _p(gpt1), gpt2.shape[0], _p(gpt2), gptm.shape[0], _p(gptm), _p(gsh), pw["step_radius"], _p(cs),
                         pw["vol"], nk, nocc, nunocc, _p(c1), _p(c2), _p(cprod),
                         cprod.shape[0] if ldc is None else ldc, col0)
    return cprod


def wfprod_pw_fft(pw, nk, nocc, nunocc, cpw_occ, cpw_unocc, nfft):
    """The FFT branch of wavefproducts2_pw (src/wavefproducts.f:576-758) in numpy:
    scatter to the grid, FFTW_BACKWARD (G -> r), conj(.)/sqrt(vol) times the step
    function, times FFT(phi_n')/nnfft, FFTW_FORWARD (r -> G), gather G_M - g.
    Returns cprod_pw (npair, ngptm). Used only to cross-check the explicit path."""
    gpt1, gpt2, gptm, gsh = pw["gpt1"], pw["gpt2"], pw["gptm"], np.asarray(pw["gshift"])
    sr = pw["step_radius"]
    ns = 2 * sr + 1
    nn = nfft ** 3
    cs = np.asarray(pw["cstep"]).reshape(ns, ns, ns, order="F")
    grid_step = np.zeros((nfft,) * 3, complex)
    for d0 in range(-sr, sr + 1):
        for d1 in range(-sr, sr + 1):
            for d2 in range(-sr, sr + 1):
                grid_step[d0 % nfft, d1 % nfft, d2 % nfft] = cs[d0 + sr, d1 + sr, d2 + sr]
    theta = np.fft.ifftn(grid_step) * nn          # FFTW_BACKWARD is unnormalised
    idx1 = tuple((gpt1 % nfft).T)
    idx2 = tuple((gpt2 % nfft).T)
    out_idx = tuple(((gptm - gsh) % nfft).T)
    c1 = np.asarray(cpw_occ).reshape(nk, nocc, gpt1.shape[0])
    c2 = np.asarray(cpw_unocc).reshape(nk, nunocc, gpt2.shape[0])
    res = np.zeros((nk, nocc, nunocc, gptm.shape[0]), complex)
    for k in range(nk):
        r1 = []
        for n in range(nocc):
            g = np.zeros((nfft,) * 3, complex)
            g[idx1] = c1[k, n]
            r1.append(np.conj(np.fft.ifftn(g) * nn / np.sqrt(pw["vol"])) * theta)
        for npr in range(nunocc):
            g = np.zeros((nfft,) * 3, complex)
            g[idx2] = c2[k, npr]
            r2 = np.fft.ifftn(g) * nn / nn
            for n in range(nocc):
                prod = np.fft.fftn(r1[n] * r2)
                res[k, n, npr] = prod[out_idx]
    # layout p = n' + nu*(n + no*k)
    return res.reshape(nk * nocc * nunocc, -1)


def trafo(cprod, ctrafo, dim=None):
    """Transform to the Coulomb eigenbasis as src/susceptibility.f:806-832 writes it for
    the complex build with FULLPW: cprod(:, :dim) = conj(matmul(conj(cprod), ctrafo))."""
    c = np.asarray(cprod)
    t = np.asarray(ctrafo)
    dim = t.shape[1] if dim is None else dim
    return np.conj(np.conj(c) @ t[:, :dim])


def olapvec(vec, gpt, cstep, sr):
    """src/overlap.f:298-316: out(i) = dotprod(row, vec) with row(j) = cstep(G_j - G_i)
    and dotprod the conjugating zdotc (src/wrapper.f:369-377); cstep on [-sr, sr]^3
    (x fastest), zero outside."""
    g = np.asarray(gpt)
    cs = np.asarray(cstep).reshape((2 * sr + 1,) * 3, order="F")
    out = np.zeros(len(g), dtype=complex)
    for i in range(len(g)):
        row = np.zeros(len(g), dtype=complex)
        for j in range(len(g)):
            d = g[j] - g[i]
            if np.all(np.abs(d) <= sr):
                row[j] = cs[d[0] + sr, d[1] + sr, d[2] + sr]
        out[i] = np.vdot(row, vec)
    return out


def trafo_olap(cprod, ctrafo, nbasp, gptm, cstep, sr, dim=None):
    """The non-FULLPW branch of src/susceptibility.f:814-824: ctrafo1 = ctrafo with its
    interstitial rows replaced by olapvec of each column, then
    cprod(:, :dim) = conj(matmul(conj(cprod), ctrafo1))."""
    t = np.array(ctrafo, dtype=complex)
    dim = t.shape[1] if dim is None else dim
    t1 = t[:, :dim].copy()
    for c in range(dim):
        t1[nbasp:, c] = olapvec(t[nbasp:, c], gptm, cstep, sr)
    return np.conj(np.conj(np.asarray(cprod)) @ t1)


def _ln(z: complex) -> complex:
    """Principal logarithm as src/hilbert.f:283-296 defines it: a real negative argument
    gives +i pi whatever the sign of its zero imaginary part."""
    import cmath
    if z.real < 0 and z.imag == 0:
        return complex(np.log(-z.real), np.pi)
    return cmath.log(z)


def getwghtS(frq, frqs, disorder=0.0, md=0, iterm=0):
    """Hilbert-transform weights of a spectral function given on the mesh frqs, for the
    frequencies frq: chi(w) = sum_s S(frqs_s) wghtS(s, w). Restates getwghtS,
    src/hilbert.f:193-281, step by step (1-based mesh indices kept as in the source;
    i = 0 is the interval before the first mesh point). Returns (wghtSr, wghtSi),
    each (nfrqs, nfrq)."""
    frq = np.asarray(frq, dtype=complex)
    frqs = np.asarray(frqs, dtype=float)
    nfrq, nfrqs = frq.size, frqs.size
    wr = np.zeros((nfrqs, nfrq))
    wi = np.zeros((nfrqs, nfrq))
    if nfrq == 0:
        return wr, wi
    F = lambda i: frqs[i - 1]                      # 1-based access
    winc = F(2) - F(1)
    a = 0.5
    if nfrqs >= 3:
        a = winc / (F(3) - F(1))
    img = 1j
    isign = -1 if iterm == 2 else 1
    while True:
        for j in range(nfrq):
            w = frq[j] * isign
            i2 = 1 if F(1) == 0 else 0
            while i2 < nfrqs:
                i1 = i2
                rdum = abs(w - F(i1 + 1))
                if rdum > min(winc / 3, 1e-6):
                    i2 = i1 + 1
                else:
                    i2 = i1 + 2
                    if i2 > nfrqs:
                        break
                w1 = max(0.0, F(i1 + 1) - a * winc) if i1 == 0 else F(i1)
                w2 = F(i2)
                int1 = int2 = 0j
                cdum = 0j
                rdum = rdum1 = rdum2 = 0.0
                if w + w1 - img * disorder != 0:
                    cdum = _ln(w - w1 + img * disorder) - _ln(w - w2 + img * disorder)
                if w1 != 0 and md > 0:
                    rdum = np.log(w2) - np.log(w1)
                    rdum1 = w2 ** -1 - w1 ** -1
                    rdum2 = (w2 ** -2 - w1 ** -2) / 2
                if md == 0:
                    int1 = cdum
                    int2 = cdum * (w + img * disorder) - (w2 - w1)
                elif md == 1:
                    int2 = cdum
                    int1 = (cdum + rdum) / (w + img * disorder) if w - img * disorder != 0 else rdum1
                elif md == 2:
                    if w - img * disorder != 0:
                        int2 = (cdum + rdum) / (w + img * disorder)
                        int1 = (int2 + rdum1) / (w + img * disorder)
                    else:
                        int2 = rdum1
                        int1 = rdum2
                if i2 - i1 == 1:
                    c = (w2 * int1 - int2) / (w2 - w1)
                    if i1 > 0:
                        wr[i1 - 1, j] += c.real
                        wi[i1 - 1, j] += c.imag
                    c = (int2 - w1 * int1) / (w2 - w1)
                    wr[i2 - 1, j] += c.real
                    wi[i2 - 1, j] += c.imag
                else:
                    if i1 > 0:
                        wr[i1 - 1, j] += isign
                    i1 += 1
                    wr[i1 - 1, j] += np.real(int1)
                    wi[i1 - 1, j] += np.imag(int1)
                    wr[i2 - 1, j] = wr[i1 - 1, j] - isign
        if iterm == 0 and isign == 1:
            isign = -1
            continue
        return wr, wi


def hilbert_weights(wtetra, wghtSr, thr=0.0, scale_all=1.0):
    """Effective imaginary-axis weights of the Hilbert-mesh path:
    w_eff(p, f) = scale_all * sum_s wtetra(p, s) wghtSr(s, f), weights <= thr dropped as
    the index lists of src/susceptibility.f:1066-1075 drop them."""
    wt = np.where(np.asarray(wtetra) > thr, wtetra, 0.0)
    return scale_all * (wt @ np.asarray(wghtSr))


def headwings(cprod, dcprod, w):
    """Head (6, nw) and wings (3, dim, nw) as the loops of src/susceptibility.f:1092-1157
    accumulate them with HILBERT NONE weights (the spectral_function sums of :1779-1782):
    head(ij, f) = sum_p dcprod(p,k1) conj(dcprod(p,k2)) w(p,f), ij = k2(k2+1)/2 + k1, k1 <= k2;
    wing(k2, i, f) = sum_p cprod(p,i) conj(dcprod(p,k2)) w(p,f)."""
    c = np.asarray(cprod)
    d = np.asarray(dcprod)
    w = np.asarray(w)
    nw = w.shape[1]
    head = np.zeros((6, nw), complex)
    for k2 in range(3):
        for k1 in range(k2 + 1):
            head[k2 * (k2 + 1) // 2 + k1] = (d[:, k1] * np.conj(d[:, k2])) @ w
    wing = np.zeros((3, c.shape[1], nw), complex)
    for k2 in range(3):
        wing[k2] = (c * np.conj(d[:, k2])[:, None]).T @ w
    return head, wing


def dielec(susceph, coul, invert=True, head=None, wing=None):
    """The dielectric matrices of src/correlation.f:614-636 from packed chi (npack, nw):
    suscep = -suscep; times sqrt(coul_i) sqrt(coul_j); plus 1 on the diagonal; then the
    inverse of each (src/correlation.f:703-745, zpptrf/zpptri). Returns the packed
    result and the transformed head (6, nw) and wing (3, nbas, nw) if given."""
    sp = np.asarray(susceph)
    npk, nw = sp.shape
    n = int(round((np.sqrt(8 * npk + 1) - 1) / 2))
    sq = np.sqrt(np.asarray(coul))
    iu, ju = np.triu_indices(n)
    idx = ju * (ju + 1) // 2 + iu
    out = np.zeros_like(sp)
    for f in range(nw):
        full = np.zeros((n, n), complex)
        full[iu, ju] = sp[idx, f]
        full[ju, iu] = np.conj(sp[idx, f])
        eps = np.eye(n) - sq[:, None] * full * sq[None, :]
        if invert:
            eps = np.linalg.inv(eps)
        out[idx, f] = eps[iu, ju]
    res = [out]
    if head is not None:
        h = -4 * np.pi * np.asarray(head)
        h[[0, 2, 5]] += 1.0
        res.append(h)
    if wing is not None:
        res.append(-np.sqrt(4 * np.pi) * sq[None, :, None] * np.asarray(wing))
    return res if len(res) > 1 else out


def chi0_realfreq(cprod, wr, wi, suscepc=None) -> np.ndarray:
    """suscepc(i, j, f) of src/susceptibility.f:1182-1235 (full-matrix layout) for real
    frequencies: per pair (i <= j) re/im = cprod(:,i) conj(cprod(:,j)) (:1199), the four
    ddots of spectral_function with wghtSr / wghtSi (:1829-1838, here the effective pair
    weights wr, wi), then
      suscepc(i,j) += cmplx(sus1, susc1) + cmplx(-susc2, sus2)
      suscepc(j,i) += cmplx(sus1, susc1) - cmplx(-susc2, sus2)   (i /= j)
    Vectorised over i for each j (numpy); returns (nbas, nbas, nw) complex."""
    cprod = np.asarray(cprod, dtype=np.complex128)
    wr = np.asarray(wr, dtype=np.float64)
    wi = np.asarray(wi, dtype=np.float64)
    npair, nbas = cprod.shape
    nw = wr.shape[1]
    if suscepc is None:
        suscepc = np.zeros((nbas, nbas, nw), dtype=np.complex128, order="F")
    for j in range(nbas):
        x = cprod[:, : j + 1] * np.conj(cprod[:, j])[:, None]      # (npair, j+1): i <= j
        re, im = x.real, x.imag
        sus1, sus2 = re.T @ wr, im.T @ wr                           # (j+1, nw)
        susc1, susc2 = re.T @ wi, im.T @ wi
        suscepc[: j + 1, j, :] += (sus1 - susc2) + 1j * (susc1 + sus2)
        lower = (sus1 + susc2) + 1j * (susc1 - sus2)
        suscepc[j, :j, :] += lower[:j]
    return suscepc


def chi0_real(cprod, w, susceph=None) -> np.ndarray:
    """The -DINV body loop (src/susceptibility.f:1182-1240 with MCOMPLEX_dp = real_dp):
    re(k) = cprod(k,i) * cprod(k,j) (:1197), sus1 = ddot(re, wghtSr(:, f)) (:1781),
    susceph(j(j+1)/2 + i, f) += sus1 (:1210), vectorised over i for each j with the
    products summed in long double. Returns (npack, nw) float64."""
    cprod = np.asarray(cprod, dtype=np.float64)
    w = np.asarray(w, dtype=np.longdouble)
    npair, nbas = cprod.shape
    nw = w.shape[1]
    if susceph is None:
        susceph = np.zeros((nbas * (nbas + 1) // 2, nw), dtype=np.float64, order="F")
    for j in range(nbas):
        re = cprod[:, : j + 1].astype(np.longdouble) * cprod[:, j].astype(np.longdouble)[:, None]
        susceph[j * (j + 1) // 2: j * (j + 1) // 2 + j + 1] += (re.T @ w).astype(np.float64)
    return susceph


def momentum_matrix(cmt_occ, cmt_unocc, cpw_occ, cpw_unocc, lcut, nrad, qmat1, qmat2, gpt, kpt,
                    rlat, cstep, sr):
    """momentum(n', n, k, x) as src/dwavefproducts.f:89-330 computes it (non-SOC, one
    atom type, nindx(l) = nrad for every l), restated loop by loop:
      F / G coefficients :135-146; MT vectors cvec1/2/3 from l+1 (qmat2, :203-219) and
      from l-1 (qmat1, :220-240); cvec(x) = dotprod(cvec_x, cmt2) / i and the Cartesian
      combination :241-253; plane waves :259-283 (vec1 = olapvec(cpw_n), qg = rlat (k+G)).
    Coefficients: cmt (nk, nb, natom, maxlm), cpw (nk, nb, ngpt). Returns
    (nunocc, nocc, nk, 3) complex."""
    nk, nocc, natom, maxlm = cmt_occ.shape
    nunocc = cmt_unocc.shape[1]
    mom = np.zeros((nunocc, nocc, nk, 3), dtype=complex)
    nlm = (lcut + 1) ** 2
    fco = np.zeros((nlm + 1, 3))
    gco = np.zeros((nlm + 1, 3))
    lm = 0
    for l in range(lcut + 1):
        for m in range(-l, l + 1):
            lm += 1
            fco[lm] = [-np.sqrt((l + m + 1) * (l + m + 2) / (2 * (2 * l + 1) * (2 * l + 3))),
                       np.sqrt((l - m + 1) * (l + m + 1) / ((2 * l + 1) * (2 * l + 3))),
                       -np.sqrt((l - m + 1) * (l - m + 2) / (2 * (2 * l + 1) * (2 * l + 3)))]
            gco[lm] = [np.sqrt(max((l - m) * (l - m - 1), 0) / (2 * (2 * l - 1) * (2 * l + 1))) if l else 0,
                       np.sqrt(max((l - m) * (l + m), 0) / ((2 * l - 1) * (2 * l + 1))) if l else 0,
                       np.sqrt(max((l + m) * (l + m - 1), 0) / (2 * (2 * l - 1) * (2 * l + 1))) if l else 0]
    q1 = np.asarray(qmat1).reshape((nrad, nrad, lcut + 1), order="F")
    q2 = np.asarray(qmat2).reshape((nrad, nrad, lcut + 1), order="F")
    for k in range(nk):
        for a in range(natom):
            for n in range(nocc):
                cmt1 = cmt_occ[k, n, a]
                cv = [np.zeros(maxlm, complex) for _ in range(3)]
                lm_0, lm_1, lm = 0, nrad, 0
                for l in range(lcut):
                    n0 = n1 = nrad
                    for m in range(-l, l + 1):
                        lm += 1
                        lm0 = lm_0 + (m + l) * n0
                        src = [lm_1 + (m + 1 + l + 1) * n1, lm_1 + (m + l + 1) * n1, lm_1 + (m - 1 + l + 1) * n1]
                        for x in range(3):
                            cv[x][lm0:lm0 + n0] = fco[lm, x] * (cmt1[src[x]:src[x] + n1] @ q2[:n1, :n0, l])
                    lm_0 += (2 * l + 1) * n0
                    lm_1 += (2 * l + 3) * n1
                lm_0, lm_1, lm = nrad, 0, 1
                for l in range(1, lcut + 1):
                    n0 = n1 = nrad
                    for m in range(-l, l + 1):
                        lm += 1
                        lm0 = lm_0 + (m + l) * n0
                        mps = [m + 1, m, m - 1]
                        for x in range(3):
                            if abs(mps[x]) <= l - 1:
                                s0 = lm_1 + (mps[x] + l - 1) * n1
                                cv[x][lm0:lm0 + n0] += gco[lm, x] * (cmt1[s0:s0 + n1] @ q1[:n1, :n0, l])
                    lm_0 += (2 * l + 1) * n0
                    lm_1 += (2 * l - 1) * n1
                for n2 in range(nunocc):
                    cmt2 = cmt_unocc[k, n2, a]
                    c = [np.vdot(cv[x], cmt2) / 1j for x in range(3)]
                    mom[n2, n, k, 0] += (c[0] - c[2]) / np.sqrt(2.0)
                    mom[n2, n, k, 1] -= (c[0] + c[2]) / np.sqrt(2.0) * 1j
                    mom[n2, n, k, 2] += c[1]
    g = np.asarray(gpt)
    for k in range(nk):
        qg = (np.asarray(rlat) @ (np.asarray(kpt[k])[:, None] + g.T)).T       # (ngpt, 3)
        for n in range(nocc):
            vec1 = olapvec(cpw_occ[k, n], g, cstep, sr)
            for n2 in range(nunocc):
                vec2 = cpw_unocc[k, n2]
                for x in range(3):
                    mom[n2, n, k, x] += np.vdot(vec1, vec2 * qg[:, x])
    return mom
