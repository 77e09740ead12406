"""numpy restatement of the cola_halo hot path -- TEST INFRASTRUCTURE.

An independent CPU statement of the reference's algorithm, used only to check
the CUDA path (tests, ``__graft_entry__.smoke()``, the CPU baseline leg of
``bench.py``).  Every function cites the reference file:line it follows.
Per-particle arithmetic is done in float32 in the reference's operation
order (so kick / drift / interpolation are bit-comparable); FFTs and mesh
sums are done in float64 (the oracle is at least as accurate as FFTW single
precision); scalar time coefficients are float64 restatements of the
reference's formulas.
"""
import math

import numpy as np
from scipy import integrate, special

f32 = np.float32
f64 = np.float64

# --------------------------------------------------------------------------
# RANLUX, 48-bit form (the RNG behind gsl_rng_ranlxd1 used at lpt.c:172-233).
# Luscher's subtract-with-borrow x_k = x_{k-5} - x_{k-12} - c (mod 1) on
# 48-bit words, 202 steps per block of 12 delivered words, 31-bit shift
# register seeding.  Vectorised over many independent streams that advance
# in lock-step (lpt.c seeds one stream per (i, j) column).
# --------------------------------------------------------------------------
_ULP48 = 1.0 / 281474976710656.0


class Ranlxd1:
    def __init__(self, seeds, luxury=202):
        seeds = np.atleast_1d(np.asarray(seeds, dtype=np.uint64)).copy()
        seeds[seeds == 0] = 1
        s = seeds & np.uint64(0xFFFFFFFF)
        ns = s.shape[0]
        bits = np.zeros((ns, 31), dtype=np.int64)
        for k in range(31):
            bits[:, k] = (s >> np.uint64(k)) & np.uint64(1)
        ib, jb = 0, 18
        x = np.zeros((ns, 12), dtype=np.float64)
        for w in range(12):
            acc = np.zeros(ns, dtype=np.float64)
            for _ in range(48):
                acc = 2.0 * acc + (bits[:, ib] ^ 1)
                bits[:, ib] ^= bits[:, jb]
                ib = (ib + 1) % 31
                jb = (jb + 1) % 31
            x[:, w] = acc * _ULP48
        self.x = x
        self.carry = np.zeros(ns, dtype=np.float64)
        self.ir, self.jr, self.ir_old = 11, 7, 0
        self.pr = luxury

    def _refill(self):
        x, carry = self.x, self.carry
        ir, jr = self.ir, self.jr
        for _ in range(self.pr):
            y = x[:, jr] - x[:, ir] - carry
            neg = y < 0.0
            carry = np.where(neg, _ULP48, 0.0)
            x[:, ir] = np.where(neg, y + 1.0, y)
            ir = (ir + 1) % 12
            jr = (jr + 1) % 12
        self.carry = carry
        self.ir, self.jr, self.ir_old = ir, jr, ir

    def uniform(self):
        self.ir = (self.ir + 1) % 12
        if self.ir == self.ir_old:
            self._refill()
        return self.x[:, self.ir].copy()


# --------------------------------------------------------------------------
# Input power spectrum (power.c:62-151) and linear growth (power.c:172-202)
# --------------------------------------------------------------------------
class PowerTable:
    def __init__(self, path):
        data = np.loadtxt(path)
        k, p = data[:, 0], data[:, 1]
        fac = 1.0 / (2.0 * math.pi * math.pi)
        self.logk = np.log10(k)                        # power.c:91
        self.logD = np.log10(fac * k * k * k * p)      # power.c:92

    def __call__(self, k):
        """PowerSpec (power.c:120-151); 0 outside the table."""
        k = np.asarray(k, dtype=np.float64)
        logk = np.log10(np.where(k > 0, k, 1.0))
        lo = np.searchsorted(self.logk, logk, side="right") - 1
        lo = np.clip(lo, 0, len(self.logk) - 2)
        hi = lo + 1
        u = (logk - self.logk[lo]) / (self.logk[hi] - self.logk[lo])
        logD = (1 - u) * self.logD[lo] + u * self.logD[hi]
        P = 10.0 ** logD / (4.0 * math.pi * k * k * k)
        out = (logk < self.logk[0]) | (logk > self.logk[-1]) | (k <= 0)
        return np.where(out, 0.0, P)

    def sigma2(self, R):
        """TopHatSigma2 (power.c:204-222): int_0^{500/R} 4 pi k^2 W^2 P dk."""
        def f(k):
            kr = R * k
            if kr < 1e-8:
                return 0.0
            w = 3 * (math.sin(kr) / kr ** 3 - math.cos(kr) / kr ** 2)
            return 4 * math.pi * k * k * w * w * float(self(k))
        edges = np.concatenate([[0.0], 10.0 ** self.logk[self.logk < math.log10(500.0 / R)],
                                [500.0 / R]])
        return sum(integrate.quad(f, a, b, epsabs=0, epsrel=1e-10, limit=200)[0]
                   for a, b in zip(edges[:-1], edges[1:]) if b > a)


def linear_growth(a, omega_m, omega_lambda=None):
    """growth(a) (power.c:177-197): H(a) int_0^a (a'/(Om + Ok a' + OL a'^3))^1.5."""
    if omega_lambda is None:
        omega_lambda = 1.0 - omega_m
    ok = 1.0 - omega_m - omega_lambda
    h = math.sqrt(omega_m / a ** 3 + ok / a ** 2 + omega_lambda)
    val = integrate.quad(lambda x: (x / (omega_m + ok * x + omega_lambda * x ** 3)) ** 1.5,
                         0.0, a, epsabs=0, epsrel=1e-13, limit=200)[0]
    return h * val


def growth_factor(astart, aend, omega_m):
    """GrowthFactor (power.c:199-202)."""
    return linear_growth(aend, omega_m) / linear_growth(astart, omega_m)


# --------------------------------------------------------------------------
# COLA time coefficients (cola.c:156-292), float64 evaluation of the
# reference formulas.  Branch decisions are taken on the single-precision
# values the reference branches on (cola.c:158-190 uses float a and x).
# --------------------------------------------------------------------------
class ColaTime:
    nLPT = -2.5        # cola.c:60

    def __init__(self, omega_m):
        self.om32 = f32(omega_m)
        self.Om = float(self.om32)     # cola.c:83  Om = Omega_m (a float)
        self._d1 = self._growth_temp(1.0)
        self._d2_1 = self._growth_d2_temp(1.0)

    def _growth_temp(self, a):
        """growthDtemp (cola.c:156-194)."""
        Om = self.Om
        a32 = f32(a)
        x32 = f32(-f64(self.om32) / (f64(self.om32) - 1.0) / f64(a32 * a32 * a32))
        x = -Om / (Om - 1.0) / (a * a * a)
        hp = hm = 0.0
        if abs(float(x32) - 1.0) < 1e-3:
            t = x - 1.0
            hp = (0.859596768064608 - 0.1016599912520404 * t + 0.025791094277821357 * t ** 2
                  - 0.008194025861121475 * t ** 3 + 0.0029076305993447644 * t ** 4
                  - 0.0011025426387159761 * t ** 5 + 0.00043707304964624546 * t ** 6
                  - 0.0001788889964687831 * t ** 7)
            hm = (1.1765206505266006 + 0.15846194123099624 * t - 0.014200487494738975 * t ** 2
                  + 0.002801728034399257 * t ** 3 - 0.0007268267888593511 * t ** 4
                  + 0.00021801569226706922 * t ** 5 - 0.00007163321597397065 * t ** 6
                  + 0.000025063737576245116 * t ** 7)
        else:
            if float(x32) < 1.0:
                hp = special.hyp2f1(0.5, 2.0 / 3.0, 5.0 / 3.0, -x)
                hm = special.hyp2f1(-0.5, 2.0 / 3.0, 5.0 / 3.0, -x)
            xi32 = f32(1.0 / f64(x32))
            xi = 1.0 / x
            if float(xi32) < 1.0 and float(xi32) > 1.0 / 30:
                hp = special.hyp2f1(-1.0 / 6.0, 0.5, 5.0 / 6.0, -xi)
                hp *= 4 * math.sqrt(xi)
                hp += -3.4494794123063873799 * xi ** (2.0 / 3.0)
                hm = special.hyp2f1(-7.0 / 6.0, -0.5, -1.0 / 6.0, -xi)
                hm *= 4.0 / 7.0 / math.sqrt(xi)
                hm += xi ** (2.0 / 3.0) * (-1.4783483195598803057)
            if float(xi32) <= 1.0 / 30.0:
                hp = (3.9999999999999996 * math.sqrt(xi) - 3.4494794123063865 * xi ** 0.6666666666666666
                      + 0.3999999999999999 * xi ** 1.5 - 0.13636363636363635 * xi ** 2.5
                      + 0.07352941176470587 * xi ** 3.5 - 0.04755434782608695 * xi ** 4.5
                      + 0.033943965517241374 * xi ** 5.5 - 0.02578125 * xi ** 6.5
                      + 0.020436356707317072 * xi ** 7.5 - 0.01671324384973404 * xi ** 8.5
                      + 0.013997779702240564 * xi ** 9.5 - 0.011945562847590041 * xi ** 10.5
                      + 0.01035003662109375 * xi ** 11.5 - 0.009080577904069926 * xi ** 12.5)
                hm = (0.5714285714285715 / math.sqrt(xi) + 2.000000000000001 * math.sqrt(xi)
                      - 1.4783483195598794 * xi ** 0.66666666666666666
                      + 0.10000000000000002 * xi ** 1.5 - 0.022727272727272735 * xi ** 2.5
                      + 0.009191176470588237 * xi ** 3.5 - 0.004755434782608697 * xi ** 4.5
                      + 0.002828663793103449 * xi ** 5.5 - 0.0018415178571428578 * xi ** 6.5
                      + 0.0012772722942073172 * xi ** 7.5 - 0.0009285135472074472 * xi ** 8.5
                      + 0.0006998889851120285 * xi ** 9.5 - 0.0005429801294359111 * xi ** 10.5
                      + 0.0004312515258789064 * xi ** 11.5 - 0.00034925299631038194 * xi ** 12.5)
        if float(a32) > 0.2:
            return math.sqrt(1.0 + (-1.0 + a ** -3) * Om) * (
                3.4494794123063873799 * (-1.0 + 1.0 / Om) ** 0.666666666666666666666666666
                + (hp * (4 * a ** 3 * (-1.0 + Om) - Om) - 7.0 * a ** 3 * hm * (-1.0 + Om))
                / (a ** 5 * (-1.0 + Om) - a ** 2 * Om))
        return (a * (1 - Om) ** 1.5 * (1291467969 * a ** 12 * (-1 + Om) ** 4
                                       + 1956769650 * a ** 9 * (-1 + Om) ** 3 * Om
                                       + 8000000000 * a ** 3 * (-1 + Om) * Om ** 3
                                       + 37490640625 * Om ** 4)) / (1.5625e10 * Om ** 5)

    def D1(self, a):
        """growthD (cola.c:196-198)."""
        return self._growth_temp(a) / self._d1

    def Q(self, a):
        """Qfactor (cola.c:201-203): a^3 H(a)/H0."""
        return math.sqrt(self.Om / (a * a * a) + 1.0 - self.Om) * a * a * a

    def _growth_d2_temp(self, a):
        d = self.D1(a)
        omega = self.Om / (self.Om + (1.0 - self.Om) * a * a * a)
        return d * d * omega ** (-1.0 / 143.0)

    def D2(self, a):
        """growthD2 (cola.c:208-216)."""
        return self._growth_d2_temp(a) / self._d2_1

    def D2v(self, a):
        """growthD2v (cola.c:219-223)."""
        omega = self.Om / (self.Om + (1.0 - self.Om) * a * a * a)
        return self.Q(a) * (self.D2(a) / a) * 2.0 * omega ** (6.0 / 11.0)

    def DprimeQ(self, a, n_growth=1.0):
        """DprimeQ (cola.c:229-234) with nDecay = 0."""
        nn = 6.0 * (1.0 - self.Om) ** 1.5 / self._d1
        decay = math.sqrt(self.Om / (a * a * a) + 1.0 - self.Om)
        d = self.D1(a)
        return decay ** -1.0 * d ** (n_growth - 1.0) * (
            n_growth * nn - (3.0 * n_growth * self.Om * d) / (2.0 * a))

    def Sq(self, ai, af, aref):
        """Sq (cola.c:262-281), fullT = 1: int a^nLPT / Q(a) da / aref^nLPT."""
        val = integrate.quad(lambda a: a ** self.nLPT / self.Q(a), ai, af,
                             epsabs=0, epsrel=1e-13, limit=200)[0]
        return val / aref ** self.nLPT

    def Sphi(self, ai, af, aref):
        """Sphi (cola.c:287-292)."""
        n = self.nLPT
        return (af ** n - ai ** n) * aref / self.Q(aref) / (n * aref ** (n - 1))

    # -- per-call coefficient sets, as the reference derives them ----------
    def kick_coeffs(self, a_v, a_x, avel1):
        """cola.c:77-91 -> (dda, q1, q2) as float32."""
        AI, A, AF = float(f32(a_v)), float(f32(a_x)), float(f32(avel1))
        om143 = (self.Om / (self.Om + (1 - self.Om) * A * A * A)) ** (1.0 / 143.0)
        dda = self.Sphi(AI, AF, A)
        g1 = self.D1(A)
        q2 = 1.5 * self.Om * g1 * g1 * (1.0 + 7.0 / 3.0 * om143)
        q1 = 1.5 * self.Om * g1
        return f32(dda), f32(q1), f32(q2)

    def drift_coeffs(self, a_x, a_v, apos1):
        """cola.c:123-134 -> (dyyy, da1, da2) as float32."""
        A, AC, AF = float(f32(a_x)), float(f32(a_v)), float(f32(apos1))
        dyyy = self.Sq(A, AF, AC)
        da1 = self.D1(AF) - self.D1(A)
        da2 = self.D2(AF) - self.D2(A)
        return f32(dyyy), f32(da1), f32(da2)


# --------------------------------------------------------------------------
# Particle updates (float32, reference operation order)
# --------------------------------------------------------------------------
def cola_kick(v, f, dx1, dx2, omega_m, dda, q1, q2):
    """cola.c:104-112.  Arrays are (n, 3) float32; returns new v."""
    om = f64(f32(omega_m))
    s = (dx1 * q1 + dx2 * q2).astype(f32)            # float products and sum
    a = ((-1.5 * om) * f.astype(f64) - s.astype(f64)).astype(f32)
    return (v + (a * dda).astype(f32)).astype(f32)


def cola_drift(x, v, dx1, dx2, dyyy, da1, da2):
    """cola.c:142-149: x += v*dyyy + (dx1*da1 + dx2*da2)."""
    lpt = (dx1 * da1 + dx2 * da2).astype(f32)
    step = ((v * dyyy).astype(f32) + lpt).astype(f32)
    return (x + step).astype(f32)


def wrap(x, boxsize):
    """move.c:34-41 (one-shot periodic wrap, per axis)."""
    L = f32(boxsize)
    x = x.copy()
    lo = x < 0
    x[lo] = (x[lo] + L).astype(f32)
    hi = (~lo) & (x >= L)
    x[hi] = (x[hi] - L).astype(f32)
    return x


# --------------------------------------------------------------------------
# PM force (pm.c:209-412) on one process: the x-direction periodicity the
# reference gets from buffer particles (pm.c:416-532) is restated exactly:
# a particle with x > L/N*N - L/N also acts through a copy at x - L.
# --------------------------------------------------------------------------
def _cic_index(x, ngrid, boxsize):
    """pm.c:230-258 for one set of positions (float32 (n,3))."""
    scale = f32(f32(ngrid) / f32(boxsize))
    X = (x[:, 0] * scale).astype(f32)
    Y = (x[:, 1] * scale).astype(f32)
    Z = (x[:, 2] * scale).astype(f32)
    iI = np.floor(X).astype(np.int64)
    J = np.trunc(Y).astype(np.int64)
    K = np.trunc(Z).astype(np.int64)
    D1 = (X - iI.astype(f32)).astype(f32)
    D2 = (Y - J.astype(f32)).astype(f32)
    D3 = (Z - K.astype(f32)).astype(f32)
    T1 = (f32(1) - D1).astype(f32)
    T2 = (f32(1) - D2).astype(f32)
    T3 = (f32(1) - D3).astype(f32)
    J = np.where(J >= ngrid, 0, J)
    K = np.where(K >= ngrid, 0, K)
    I1 = iI + 1
    J1 = np.where(J + 1 >= ngrid, 0, J + 1)
    K1 = np.where(K + 1 >= ngrid, 0, K + 1)
    return iI, I1, J, J1, K, K1, D1, D2, D3, T1, T2, T3


def buffer_copies(x, ngrid, boxsize):
    """send_buffer_positions (pm.c:416-502) on one rank: indices and shifted
    positions of the buffer particles."""
    L = f32(boxsize)
    eps = f32(L / f32(ngrid))
    x_right = f32(f32(eps * f32(ngrid)) - eps)
    sel = np.nonzero(x[:, 0] > x_right)[0]
    g = x[sel].copy()
    g[:, 0] = (g[:, 0] + f32(-L)).astype(f32)
    return sel, g


def cic_deposit(x, ngrid, boxsize, factor):
    """PtoMesh (pm.c:209-276): delta = -1 + factor^3 sum CIC, float64 sums.

    Returns an (N, N, N) float64 mesh."""
    N = ngrid
    sel, g = buffer_copies(x, ngrid, boxsize)
    pos = np.concatenate([x, g])
    wpar = f32(f32(factor) ** 3)
    iI, I1, J, J1, K, K1, D1, D2, D3, T1, T2, T3 = _cic_index(pos, N, boxsize)
    T2W = (T2 * wpar).astype(f32)
    D2W = (D2 * wpar).astype(f32)
    mesh = np.zeros(N * N * N, dtype=np.float64)

    def put(ix, jy, kz, w, ok):
        # float64 sums per cell (bincount: the same sums as a sequential
        # scatter up to float64 rounding, and fast at 768^3)
        idx = (ix[ok] * N + jy[ok]) * N + kz[ok]
        mesh[:] += np.bincount(idx, weights=w[ok].astype(np.float64), minlength=N * N * N)

    ok0 = (iI >= 0) & (iI < N)
    ok1 = (I1 >= 0) & (I1 < N)
    put(iI, J, K, ((T3 * T1).astype(f32) * T2W).astype(f32), ok0)
    put(iI, J, K1, ((D3 * T1).astype(f32) * T2W).astype(f32), ok0)
    put(iI, J1, K, ((T3 * T1).astype(f32) * D2W).astype(f32), ok0)
    put(iI, J1, K1, ((D3 * T1).astype(f32) * D2W).astype(f32), ok0)
    put(I1, J, K, ((T3 * D1).astype(f32) * T2W).astype(f32), ok1)
    put(I1, J, K1, ((D3 * D1).astype(f32) * T2W).astype(f32), ok1)
    put(I1, J1, K, ((T3 * D1).astype(f32) * D2W).astype(f32), ok1)
    put(I1, J1, K1, ((D3 * D1).astype(f32) * D2W).astype(f32), ok1)
    return mesh.reshape(N, N, N) - 1.0


def r2c(real):
    """Unnormalised 3-D r2c (FFTW convention), half spectrum on the last axis."""
    return np.fft.rfftn(real.astype(np.float64))


def c2r(half, n):
    """Unnormalised 3-D c2r with FFTW's treatment of a non-Hermitian input:
    c2c over the first two axes, then a 1-D c2r over the last axis that uses
    only the real parts of its k=0 and k=n/2 coefficients."""
    g = np.fft.ifftn(half.astype(np.complex128), axes=(0, 1), norm="forward")
    g[:, :, 0] = g[:, :, 0].real
    if n % 2 == 0:
        g[:, :, n // 2] = g[:, :, n // 2].real
    return np.fft.irfft(g, n=n, axis=2, norm="forward")


def filter_at(den, knots, ngrid):
    """Force transfer function T(|n|) at |n|^2 = den (no reference
    counterpart: the Fourier-space learned correction of libcolagpu): knots
    equally spaced over 0 <= |n| <= sqrt(3) ngrid / 2, linear in between,
    float32 arithmetic in the device's order."""
    t = np.asarray(knots, dtype=f32)
    n = len(t)
    inv_dn = f32((n - 1) / (math.sqrt(3.0) * ngrid / 2.0))
    r = (np.sqrt(den.astype(f32)).astype(f32) * inv_dn).astype(f32)
    i = r.astype(np.int64)
    last = i >= n - 1
    ic = np.minimum(i, n - 2)
    a, b = t[ic], t[ic + 1]
    v = (a + ((r - ic.astype(f32)).astype(f32) * (b - a).astype(f32)).astype(f32)).astype(f32)
    return np.where(last, t[n - 1], v).astype(f32)


def force_kernel_tables(ngrid, gradient=0, laplacian=0, deconvolve=0):
    """Per-axis tables of the Green step's options (no reference
    counterpart; libcolagpu's cg_sim_set_force_kernel), float32 from float64
    formulas, indexed by the FFT index i (signed s = i <= N/2 ? i : i - N):
    gradient factor (s; 2-point N/2pi sin 2w; 4-point N/2pi (8 sin 2w -
    sin 4w)/6, w = pi s/N), Laplacian term (s^2 or (N/pi sin w)^2) and the
    CIC window correction sinc(w)^(-2 deconvolve)."""
    N = ngrid
    i = np.arange(N)
    s = np.where(i <= N // 2, i, i - N).astype(np.float64)
    w = np.pi * s / N
    if gradient == 2:
        g = N / (2 * np.pi) * np.sin(2 * w)
    elif gradient == 4:
        g = N / (2 * np.pi) * (8 * np.sin(2 * w) - np.sin(4 * w)) / 6
    else:
        g = s
    lap = (N / np.pi * np.sin(w)) ** 2 if laplacian else s * s
    sinc = np.where(i == 0, 1.0, np.sin(w) / np.where(w == 0, 1.0, w))
    c = (sinc * sinc) ** (-float(deconvolve))
    return g.astype(f32), lap.astype(f32), c.astype(f32)


def force_spectrum(delta_k, ngrid, boxsize, axis, knots=None, kernel=(0, 0, 0)):
    """compute_force_mesh (pm.c:304-346): F = i f2 delta_k,
    f2 = f1 n_axis / |n|^2, f1 = -1/(N^3 * 2 pi/L), signed frequencies with
    the Nyquist index kept at +N/2 for x and y; F(0) = 0.  Beyond the
    reference: `knots` multiplies f2 by filter_at(|n|^2) before n_axis, and
    kernel = (gradient, laplacian, deconvolve) replaces n_axis, |n|^2 and
    the window factor by force_kernel_tables' entries, in the device's
    float32 order."""
    N = ngrid
    scale = f32(2.0 * math.pi / f64(f32(boxsize)))
    f1 = f32(-1.0 / N ** 3 / f64(scale))
    idx = np.arange(N)
    s = np.where(idx <= N // 2, idx, idx - N)
    I0 = s[:, None, None]
    J0 = s[None, :, None]
    K = np.arange(N // 2 + 1)[None, None, :]
    den = (K * K + I0 * I0 + J0 * J0)
    den = np.where(den == 0, 1, den)
    di = [I0, J0, K][axis]
    if tuple(kernel) == (0, 0, 0):
        g = (f1 / den.astype(f32)).astype(f32)
        if knots is not None:
            g = (g * filter_at(den, knots, N)).astype(f32)
        f2 = (g * np.asarray(di, dtype=f32)).astype(f32)
    else:
        gt, lt, wt = force_kernel_tables(N, *kernel)
        ix = idx[:, None, None]
        iy = idx[None, :, None]
        iz = np.arange(N // 2 + 1)[None, None, :]
        dl = ((lt[ix] + lt[iy]).astype(f32) + lt[iz]).astype(f32)
        g = (f1 / np.where(dl == 0, f32(1), dl)).astype(f32)
        if knots is not None:
            g = (g * filter_at(den, knots, N)).astype(f32)
        g = (g * ((wt[ix] * wt[iy]).astype(f32) * wt[iz]).astype(f32)).astype(f32)
        f2 = (g * [gt[ix], gt[iy], gt[iz]][axis]).astype(f32)
    F = 1j * f2.astype(np.float64) * delta_k
    F[0, 0, 0] = 0.0
    return F


def pm_force_meshes(x, ngrid, boxsize, factor, knots=None, kernel=(0, 0, 0)):
    """Density, check sum and the three real force meshes (float64)."""
    dens = cic_deposit(x, ngrid, boxsize, factor)
    dk = r2c(dens)
    meshes = [c2r(force_spectrum(dk, ngrid, boxsize, a, knots, kernel), ngrid)
              for a in range(3)]
    return dens, dk, meshes


def cic_interp(x, mesh32, ngrid, boxsize):
    """force_at_particle_locations (pm.c:359-412) for one component, float32
    arithmetic in the reference's order, plus the buffer-particle force added
    back by add_buffer_forces (pm.c:526-531)."""
    N = ngrid

    def interp(pos):
        iI, I1, J, J1, K, K1, D1, D2, D3, T1, T2, T3 = _cic_index(pos, N, boxsize)
        m = mesh32
        f = np.zeros(pos.shape[0], dtype=f32)
        ok0 = (iI >= 0) & (iI < N)
        ok1 = (I1 >= 0) & (I1 < N)
        i0 = np.where(ok0, iI, 0)
        i1 = np.where(ok1, I1, 0)

        def term(ix, jy, kz, wa, wb, wc):
            return (((m[ix, jy, kz] * wa).astype(f32) * wb).astype(f32) * wc).astype(f32)
        a = (((term(i0, J, K, T3, T1, T2) + term(i0, J, K1, D3, T1, T2)).astype(f32)
              + term(i0, J1, K, T3, T1, D2)).astype(f32) + term(i0, J1, K1, D3, T1, D2)).astype(f32)
        b = (((term(i1, J, K, T3, D1, T2) + term(i1, J, K1, D3, D1, T2)).astype(f32)
              + term(i1, J1, K, T3, D1, D2)).astype(f32) + term(i1, J1, K1, D3, D1, D2)).astype(f32)
        f = np.where(ok0, (f + a).astype(f32), f)
        f = np.where(ok1, (f + b).astype(f32), f)
        return f

    f = interp(x)
    sel, g = buffer_copies(x, ngrid, boxsize)
    if sel.size:
        fg = interp(g)
        f[sel] = (f[sel] + fg).astype(f32)
    return f


def pm_calculate_forces(x, ngrid, boxsize, factor, knots=None, kernel=(0, 0, 0)):
    """pm_calculate_forces (pm.c:565-596): (n,3) float32 forces."""
    dens, dk, meshes = pm_force_meshes(x, ngrid, boxsize, factor, knots, kernel)
    f = np.stack([cic_interp(x, m.astype(f32), ngrid, boxsize) for m in meshes], axis=1)
    return f.astype(f32), dens


def check_total_density(dens, factor, np_total):
    """check_total_density (pm.c:535-562): (sum, tolerance, ok)."""
    s = float(np.sum(dens, dtype=np.float64))
    tol = 1.0e-7 * factor ** 3 * np_total
    return s, tol, abs(s) <= tol


# --------------------------------------------------------------------------
# 2LPT initial displacements (lpt.c:145-578), one process.
# --------------------------------------------------------------------------
def _seedtable(seed, N):
    """lpt.c:172-207."""
    r = Ranlxd1([seed])
    st = np.zeros((N, N), dtype=np.uint64)

    def draw():
        return np.uint64(int(0x7fffffff * float(r.uniform()[0])))
    for i in range(N // 2):
        for j in range(i):
            st[i, j] = draw()
        for j in range(i + 1):
            st[j, i] = draw()
        for j in range(i):
            st[N - 1 - i, j] = draw()
        for j in range(i + 1):
            st[N - 1 - j, i] = draw()
        for j in range(i):
            st[i, N - 1 - j] = draw()
        for j in range(i + 1):
            st[j, N - 1 - i] = draw()
        for j in range(i):
            st[N - 1 - i, N - 1 - j] = draw()
        for j in range(i + 1):
            st[N - 1 - j, N - 1 - i] = draw()
    return st


def lpt_modes(N, seed):
    """Per-column RNG draws (lpt.c:219-233): phase and amplitude arrays of
    shape (N, N, N/2) and the seed table."""
    st = _seedtable(seed, N)
    r = Ranlxd1(st.reshape(-1))
    phase = np.zeros((N * N, N // 2))
    ampl = np.zeros((N * N, N // 2))
    for k in range(N // 2):
        phase[:, k] = r.uniform() * 2 * math.pi
        a = r.uniform()
        if np.any(a == 0.0):
            raise NotImplementedError("ampl == 0 retry (probability 2^-48)")
        ampl[:, k] = a
    return phase.reshape(N, N, N // 2), ampl.reshape(N, N, N // 2), st


def lpt_za_spectrum(N, boxsize, seed, power):
    """cdisp[3] of lpt.c:210-351 as complex128 arrays (3, N, N, N/2+1)."""
    phase, ampl, _ = lpt_modes(N, seed)
    fac = (2 * math.pi / boxsize) ** 1.5
    idx = np.arange(N)
    kv = np.where(idx < N // 2, idx, -(N - idx)) * 2 * math.pi / boxsize
    kx = kv[:, None, None]
    ky = kv[None, :, None]
    kz = (np.arange(N // 2) * 2 * math.pi / boxsize)[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    kmag = np.sqrt(k2)
    valid = np.ones((N, N, N // 2), dtype=bool)
    valid[N // 2, :, :] = False
    valid[:, N // 2, :] = False
    valid[0, 0, 0] = False
    k2s = np.where(valid, k2, 1.0)
    p = np.where(valid, power(np.where(valid, kmag, 1.0)), 0.0) * -np.log(ampl)
    delta = fac * np.sqrt(p)
    disp = np.zeros((3, N, N, N // 2 + 1), dtype=np.complex128)
    kvecs = [np.broadcast_to(kx, k2.shape), np.broadcast_to(ky, k2.shape),
             np.broadcast_to(kz, k2.shape)]
    for a in range(3):
        re = -kvecs[a] / k2s * delta * np.sin(phase)
        im = kvecs[a] / k2s * delta * np.cos(phase)
        val = np.where(valid, re + 1j * im, 0.0)
        # k > 0 (lpt.c:278-288)
        disp[a, :, :, 1:N // 2] = val[:, :, 1:]
        # k = 0 plane (lpt.c:289-347)
        for j in range(1, N // 2):
            v = val[0, j, 0]
            disp[a, 0, j, 0] = v
            disp[a, 0, N - j, 0] = v.real - 1j * v.imag
        for i in range(1, N // 2):
            for j in range(N):
                if not valid[i, j, 0]:
                    continue
                v = val[i, j, 0]
                disp[a, i, j, 0] = v
                disp[a, N - i, (N - j) % N, 0] = v.real - 1j * v.imag
    return disp


def lpt_set_displacement(N, boxsize, seed, omega_m, a_init, power):
    """lpt.c:145-578 -> dict of float32 particle arrays in lattice order."""
    disp_k = lpt_za_spectrum(N, boxsize, seed, power)
    idx = np.arange(N)
    kv = np.where(idx < N // 2, idx, -(N - idx)) * 2 * math.pi / boxsize
    kx = kv[:, None, None]
    ky = kv[None, :, None]
    kz = np.where(np.arange(N // 2 + 1) < N // 2, np.arange(N // 2 + 1),
                  -(N - np.arange(N // 2 + 1)))[None, None, :] * 2 * math.pi / boxsize
    kk = [kx, ky, kz]
    # lpt.c:358-398 gradients i k_j disp_i: (0,0)(0,1)(0,2)(1,1)(1,2)(2,2)
    pairs = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    grad = [c2r(1j * kk[j] * disp_k[i], N) for i, j in pairs]
    src = (grad[0] * (grad[3] + grad[5]) + grad[3] * grad[5]
           - grad[1] ** 2 - grad[2] ** 2 - grad[4] ** 2)   # lpt.c:414-419
    S = r2c(src)
    k2 = kx * kx + ky * ky + kz * kz
    disp2_k = []
    for a in range(3):
        d = np.where(k2 > 0, -1j * kk[a] / np.where(k2 > 0, k2, 1.0) * S, 0.0)  # lpt.c:479-486
        disp2_k.append(d)
    dis = np.stack([c2r(disp_k[a], N) for a in range(3)], axis=-1).astype(f32)
    dis2 = np.stack([c2r(disp2_k[a], N) for a in range(3)], axis=-1)
    dis2 = (dis2 * (1.0 / float(N) ** 3)).astype(f32)                # lpt.c:541
    dplus = 1.0 / growth_factor(a_init, 1.0, omega_m)                  # lpt.c:509
    om = omega_m / (omega_m + (1.0 - omega_m) * a_init ** 3)
    D2 = dplus * dplus * (om / omega_m) ** (-1.0 / 143.0)
    D20 = omega_m ** (-1.0 / 143.0)
    dx = f32(boxsize / N)
    q = ((np.arange(N).astype(f32) + f32(0.5)) * dx).astype(f32)
    Q = np.stack(np.meshgrid(q, q, q, indexing="ij"), axis=-1)
    x = (Q.astype(f64) + dis.astype(f64) * dplus
         - 3.0 / 7.0 * D20 * dis2.astype(f64) * D2).astype(f32)
    dx2 = (-3.0 / 7.0 * D20 * dis2.astype(f64)).astype(f32)
    n = N ** 3
    return {
        "x": x.reshape(n, 3), "dx1": dis.reshape(n, 3), "dx2": dx2.reshape(n, 3),
        "v": np.zeros((n, 3), dtype=f32), "id": np.arange(1, n + 1, dtype=np.int64),
        "dplus": dplus, "D2": D2,
    }


# --------------------------------------------------------------------------
# Power spectrum estimator (no reference counterpart): shell average of
# |delta_k|^2 in linear bins of width dk = 2 pi/L, modes 0 < kz < N/2 counted
# twice (Hermitian half spectrum).
# --------------------------------------------------------------------------
def power_spectrum(delta, boxsize, nbins=None, deconvolve_cic=False):
    N = delta.shape[0]
    try:   # the same float64 transform, on all host threads where scipy has them
        import scipy.fft
        dk = scipy.fft.rfftn(delta.astype(np.float64), workers=-1)
    except ImportError:
        dk = np.fft.rfftn(delta.astype(np.float64))
    dk /= N ** 3
    kf = 2 * math.pi / boxsize
    idx = np.arange(N)
    s = np.where(idx <= N // 2, idx, idx - N)
    nz = np.arange(N // 2 + 1)

    def w(n):
        x = math.pi * n / N
        return np.where(n == 0, 1.0, np.sin(x) / np.where(n == 0, 1.0, x)) ** 2
    if nbins is None:
        nbins = N // 2
    cnt = np.zeros(nbins + 1)
    ps = np.zeros(nbins + 1)
    ks = np.zeros(nbins + 1)
    # one kx plane at a time (bounded memory at 768^3)
    for i in range(N):
        n2 = s[i] ** 2 + s[:, None] ** 2 + nz[None, :] ** 2
        kmag = np.sqrt(n2) * kf
        p = np.abs(dk[i]) ** 2 * boxsize ** 3
        if deconvolve_cic:
            p = p / (w(s[i]) * w(s)[:, None] * w(nz)[None, :]) ** 2
        wgt = np.where((nz == 0) | (nz == N // 2), 1.0, 2.0)[None, :] * np.ones_like(kmag)
        ib = np.floor(kmag / kf + 0.5).astype(np.int64)   # bin i: |n| in [i-1/2, i+1/2)
        ok = (ib >= 1) & (ib <= nbins)
        cnt += np.bincount(ib[ok], weights=wgt[ok], minlength=nbins + 1)
        ps += np.bincount(ib[ok], weights=(wgt * p)[ok], minlength=nbins + 1)
        ks += np.bincount(ib[ok], weights=(wgt * kmag)[ok], minlength=nbins + 1)
    cnt, ps, ks = cnt[1:], ps[1:], ks[1:]
    with np.errstate(invalid="ignore", divide="ignore"):
        return ks / cnt, ps / cnt, cnt


def cola_set_snapshot(x, v, f, dx1, dx2, a_x, a_v, aout, ct):
    """cola_set_snapshot (cola.c:341-410): final kick + drift into a snapshot,
    velocities in km/s with the 2LPT velocity added back.  Returns (x, v)."""
    vfac = f32(100.0 / aout)
    A, AI, AF = float(f32(a_x)), float(f32(a_v)), float(f32(aout))
    dda, q1, q2 = ct.kick_coeffs(AI, A, AF)
    Dv = f32(ct.DprimeQ(AF, 1.0))
    Dv2 = f32(ct.D2v(AF))
    dyyy, da1, da2 = ct.drift_coeffs(A, AI, AF)
    om = f64(f32(ct.Om))
    s = (dx1 * q1 + dx2 * q2).astype(f32)
    acc = ((-1.5 * om) * f.astype(f64) - s.astype(f64)).astype(f32)
    vel = (v + (acc * dda).astype(f32)).astype(f32)
    vel = (vel + (dx1 * Dv + dx2 * Dv2).astype(f32)).astype(f32)
    vel = (vfac * vel).astype(f32)
    pos = (x + (v * dyyy).astype(f32)).astype(f32)
    pos = (pos + (dx1 * da1 + dx2 * da2).astype(f32)).astype(f32)
    return pos, vel


class OracleRun:
    """The reference time loop (main.c:117-206) on restated kernels."""

    def __init__(self, ngrid, boxsize, factor, omega_m, x, dx1, dx2, a_init):
        self.ngrid, self.L, self.factor = ngrid, boxsize, factor
        self.ct = ColaTime(omega_m)
        self.omega_m = omega_m
        self.x = x.astype(f32).copy()
        self.dx1 = dx1.astype(f32).copy()
        self.dx2 = dx2.astype(f32).copy()
        self.v = np.zeros_like(self.x)
        self.f = np.zeros_like(self.x)
        self.a_x = f32(a_init)
        self.a_v = f32(a_init)
        self.snapshots = []

    def move(self):
        self.x = wrap(self.x, self.L)

    def force(self):
        self.f, _ = pm_calculate_forces(self.x, self.ngrid, self.L, self.factor)

    def kick(self, avel1):
        dda, q1, q2 = self.ct.kick_coeffs(self.a_v, self.a_x, avel1)
        self.v = cola_kick(self.v, self.f, self.dx1, self.dx2, self.omega_m, dda, q1, q2)
        self.a_v = f32(avel1)

    def drift(self, apos1):
        dyyy, da1, da2 = self.ct.drift_coeffs(self.a_x, self.a_v, apos1)
        self.x = cola_drift(self.x, self.v, self.dx1, self.dx2, dyyy, da1, da2)
        self.a_x = f32(apos1)

    def snapshot(self, aout, iout):
        pos, vel = cola_set_snapshot(self.x, self.v, self.f, self.dx1, self.dx2,
                                     self.a_x, self.a_v, aout, self.ct)
        self.snapshots.append((aout, pos, vel))


# --------------------------------------------------------------------------
# Friends-of-friends halos (fof.c:427-1181 on one rank).
def fof_halos(x, v, boxsize, ll, nfof_min=32):
    """Periodic friends-of-friends: particles closer than `ll` (strict,
    squared distance in float32 as kdFoF forms it, fof.c:569-572) are
    linked; groups of at least nfof_min (fof.c:224) are halos.  Positions
    are wrapped into the box first (move_particles2_min, fof.c:1042).
    Returns rows (nfof, x[3], v[3]) with the halo centre = one member plus
    the mean minimum-image offset of all members, wrapped into [0, L)
    (fof.c:287-322, 1141-1150), and the mean velocity; sorted by
    (nfof, x, y, z)."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    from scipy.spatial import cKDTree
    L = f32(boxsize)
    x = wrap(np.asarray(x, dtype=f32), L)
    n = len(x)
    if n == 0:
        return np.zeros((0, 7))
    # candidates within ll (inclusive, in float64), then the float32 test
    xs = np.where(x >= L, np.nextafter(L, f32(0)), x).astype(np.float64)
    tree = cKDTree(xs, boxsize=float(L) + 1e-9)
    pairs = tree.query_pairs(r=float(ll) * (1 + 1e-6), output_type="ndarray")
    keep = np.zeros(len(pairs), dtype=bool)
    if len(pairs):
        a, b = pairs[:, 0], pairs[:, 1]
        d = x[a] - x[b]
        half = f32(0.5) * L
        d = np.where(d > half, (x[a] - L) - x[b], np.where(d < -half, (x[b] - L) - x[a], d))
        d = d.astype(f32)
        d2 = ((d[:, 0] * d[:, 0]).astype(f32) + (d[:, 1] * d[:, 1]).astype(f32)).astype(f32)
        d2 = (d2 + (d[:, 2] * d[:, 2]).astype(f32)).astype(f32)
        keep = d2 < f32(ll) * f32(ll)
        pairs = pairs[keep]
    g = coo_matrix((np.ones(len(pairs)), (pairs[:, 0], pairs[:, 1])), shape=(n, n))
    ncomp, lab = connected_components(g, directed=False)
    sizes = np.bincount(lab, minlength=ncomp)
    rows = []
    v = np.asarray(v, dtype=np.float64)
    for c in np.nonzero(sizes >= nfof_min)[0]:
        idx = np.nonzero(lab == c)[0]
        x0 = x[idx[0]].astype(np.float64)
        dx = x[idx].astype(np.float64) - x0
        dx = np.where(dx > 0.5 * float(L), dx - float(L), np.where(dx < -0.5 * float(L), dx + float(L), dx))
        c0 = x0 + dx.mean(axis=0)
        c0 = np.where(c0 < 0, c0 + float(L), c0)
        c0 = np.where(c0 >= float(L), c0 - float(L), c0)
        rows.append([len(idx), *c0, *v[idx].mean(axis=0)])
    rows = np.array(rows).reshape(-1, 7)
    order = np.lexsort((rows[:, 3], rows[:, 2], rows[:, 1], rows[:, 0]))
    return rows[order]


# --------------------------------------------------------------------------
# Coarse density grid (coarse_grid.c:17-121 on one rank).
def coarse_grid(x, boxsize, nc, np_total=None):
    """CIC density contrast on an nc^3 grid [x][y][z].  Float32 throughout in
    the reference's operation order: s = x * (nc / L), ix = floor(s), left
    weight w = 1 - (s - ix), periodic neighbours (coarse_grid.c:96-108), the
    eight products formed left to right and added particle by particle,
    corner by corner (coarse_grid.c:110-120); then delta = nbar_inv * rho - 1
    with nbar_inv = (double) nc^3 / np_total rounded to float
    (coarse_grid.c:51, 70-73).  Returns (delta, sum of rho in float64)."""
    x = np.asarray(x, dtype=f32).reshape(-1, 3)
    n = len(x)
    ng = nc * nc * nc
    dx_inv = f32(nc) / f32(boxsize)
    s = x * dx_inv
    ix = np.floor(s).astype(np.int64)
    w = f32(1.0) - (s - ix.astype(f32))
    u = f32(1.0) - w
    i0 = np.mod(ix, nc)
    i1 = np.mod(ix + 1, nc)
    # corner order of coarse_grid.c:113-120: (x, y, z) from {0: left, 1: right}
    corners = ((0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1),
               (1, 0, 0), (1, 1, 0), (1, 0, 1), (1, 1, 1))
    idx = np.empty((n, 8), dtype=np.int64)
    val = np.empty((n, 8), dtype=f32)
    for c, (a, b, d) in enumerate(corners):
        ia = i1[:, 0] if a else i0[:, 0]
        ib = i1[:, 1] if b else i0[:, 1]
        id_ = i1[:, 2] if d else i0[:, 2]
        wa = u[:, 0] if a else w[:, 0]
        wb = u[:, 1] if b else w[:, 1]
        wd = u[:, 2] if d else w[:, 2]
        idx[:, c] = (ia * nc + ib) * nc + id_
        val[:, c] = (wa * wb) * wd
    grid = np.zeros(ng, dtype=f32)
    np.add.at(grid, idx.ravel(), val.ravel())       # sequential, in order
    total = float(np.sum(grid, dtype=f64))
    nbar_inv = f32(float(ng) / float(n if np_total is None else np_total))
    delta = nbar_inv * grid - f32(1.0)
    return delta.reshape(nc, nc, nc), total


# --------------------------------------------------------------------------
# GADGET-1 snapshot file (write.c:14-107 on one rank).
def gadget_bytes(x, v, ids, a, boxsize, omega_m, h, use_long_id=False, np_total=None,
                 num_files=1):
    """The file as bytes: four records, each framed by its int32 byte length
    -- the 256-byte header (gadget_file.h:4-24), positions, velocities times
    vfac = (float)(1/sqrt(a)) in float32, ids as uint32 (or uint64 with
    use_long_id).  Header values are formed in float64 from the float32
    snapshot fields as write.c:42-64 forms them."""
    import struct
    x = np.asarray(x, dtype=f32).reshape(-1, 3)
    v = np.asarray(v, dtype=f32).reshape(-1, 3)
    ids = np.asarray(ids, dtype=np.int64)
    n = len(x)
    nt = n if np_total is None else int(np_total)
    L, om, af, hf = (float(f32(boxsize)), float(f32(omega_m)), float(f32(a)), float(f32(h)))
    with np.errstate(divide="ignore", invalid="ignore"):   # C: n = 0 gives inf
        mass = float(f64(om * 27.7455 * math.pow(L, 3.0)) / f64(nt))
    hdr = struct.pack("<6i6d2d2i6I2i4d2i6Ii", 0, n, 0, 0, 0, 0,
                      0.0, mass, 0.0, 0.0, 0.0, 0.0,
                      af, 1.0 / af - 1, 0, 0,
                      0, nt & 0xFFFFFFFF, 0, 0, 0, 0,
                      0, num_files, L, om, 1.0 - om, hf, 0, 0,
                      0, (nt >> 32) & 0xFFFFFFFF, 0, 0, 0, 0, 0)
    hdr += b"\0" * (256 - len(hdr))
    assert len(hdr) == 256
    vfac = f32(1.0 / math.sqrt(af))
    vel = (vfac * v).astype(f32)
    idarr = ids.astype(np.uint64) if use_long_id else (ids & 0xFFFFFFFF).astype(np.uint32)

    def rec(payload):
        m = struct.pack("<i", len(payload) & 0xFFFFFFFF if len(payload) < 2 ** 31
                        else len(payload) - 2 ** 32)
        return m + payload + m
    return (rec(hdr) + rec(x.tobytes()) + rec(vel.tobytes()) + rec(idarr.tobytes()))
