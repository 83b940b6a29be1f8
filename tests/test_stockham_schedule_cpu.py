"""CPU model of the Stockham schedule of csrc/fft_smem.cuh (Sched, PassShape,
pass_load / pass_store index arithmetic, the 3 * 2^a register FFTs) checked
against NumPy's FFT for every line length the kernels use: 2^k, 3 * 2^k with
24 values per thread and the wide 3 * 2^k form with 48 values per thread.
Also checks that every pass gives each thread V values (the static_assert of
PassShape), that the stores of a pass cover the line exactly once, and that
the twiddle tables fit the slots the handles allocate for them (forward
table at offset 0 and reversed table at 3L/2 in the propagator, at 2L in the
FBP and Paganin handles, 2L entries in the Radon handle)."""
import numpy as np
import pytest


def sched(L, rev=False, wide=False):
    """(P, G, V, radices) as stockham::Sched<L, rev, wide ? 48 : 0>."""
    p2 = (L & (L - 1)) == 0
    assert p2 or (L % 3 == 0 and ((L // 3) & (L // 3 - 1)) == 0)
    k2 = int(np.log2(L if p2 else L // 3))
    w = wide and not p2
    base = 16 if (p2 or w) else 8
    vb = 16 if p2 else (48 if w else 24)
    P = ((1 if L <= 16 else (k2 + 3) // 4) if p2 else (1 + k2 // 4 if w else 1 + k2 // 3))
    G = L // vb if L >= vb else 1
    V = vb if L >= vb else L
    small = (L >> (4 * (P - 1))) if (p2 or w) else (L >> (3 * (P - 1)))
    rad = [(small if p == 0 else base) if rev else (base if p < P - 1 else small) for p in range(P)]
    return P, G, V, rad


def reg_fft(v, inv):
    """The register FFTs: radix 2^a directly, R = 3M as a 3-point DFT over
    n1 (n = M n1 + n2), the twiddle W_R^(n2 k1), then M-point FFTs over n2
    (X[k1 + 3 k2])."""
    R = len(v)
    if R % 3:
        return np.fft.ifft(v) * R if inv else np.fft.fft(v)
    M = R // 3
    h = np.sqrt(3) / 2 * (-1 if inv else 1)
    y = np.zeros((3, M), complex)
    for n2 in range(M):
        a, b, c = v[n2], v[M + n2], v[2 * M + n2]
        t, d = b + c, b - c
        m = a - 0.5 * t
        y[0, n2] = a + t
        y1 = complex(m.real + h * d.imag, m.imag - h * d.real)
        y2 = complex(m.real - h * d.imag, m.imag + h * d.real)
        w = np.exp((1 if inv else -1) * 2j * np.pi * n2 * np.array([1, 2]) / R)
        y[1, n2], y[2, n2] = y1 * w[0], y2 * w[1]
    out = np.zeros(R, complex)
    for k1 in range(3):
        yy = np.fft.ifft(y[k1]) * M if inv else np.fft.fft(y[k1])
        out[k1 + 3 * np.arange(M)] = yy
    return out


def run(x, rev, inv, wide):
    L = len(x)
    P, G, V, rad = sched(L, rev, wide)
    src, ns = x.astype(complex), 1
    for p in range(P):
        RP = rad[p]
        NG = L // RP
        Q = NG // G
        assert Q * G == NG and Q * RP == V, (L, p, RP)
        dst, seen = np.zeros(L, complex), np.zeros(L, int)
        for t in range(G):
            for q in range(Q):
                j = t + G * q
                v = src[j + np.arange(RP) * NG]
                k = j % ns
                if ns > 1:
                    v = v * np.exp((1 if inv else -1) * 2j * np.pi * np.arange(RP) * k / (ns * RP))
                X = reg_fft(v, inv)
                pos = (j // ns) * ns * RP + k + np.arange(RP) * ns
                dst[pos] = X
                seen[pos] += 1
        assert (seen == 1).all()
        src, ns = dst, ns * RP
    return src


def tw_size(L, rev, wide=False):
    P, G, V, rad = sched(L, rev, wide)
    o, ns = 0, rad[0]
    for p in range(1, P):
        o += ns * rad[p]
        ns *= rad[p]
    return o


LENGTHS = [3, 6, 12, 24, 48, 96, 192, 384, 768, 1536, 3072, 6144, 16, 32, 64, 512, 2048, 4096]


@pytest.mark.parametrize("L", LENGTHS)
def test_schedule_matches_numpy(L):
    rng = np.random.default_rng(L)
    x = rng.standard_normal(L) + 1j * rng.standard_normal(L)
    for rev in (False, True):
        for inv in (False, True):
            ref = np.fft.ifft(x) * L if inv else np.fft.fft(x)
            got = run(x, rev, inv, False)
            assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()


@pytest.mark.parametrize("L", [6144, 12288])
def test_wide_schedule_matches_numpy(L):
    rng = np.random.default_rng(L)
    x = rng.standard_normal(L) + 1j * rng.standard_normal(L)
    P, G, V, rad = sched(L, False, True)
    assert V == 48 and rad[0] == 16
    for inv in (False, True):
        ref = np.fft.ifft(x) * L if inv else np.fft.fft(x)
        assert np.abs(run(x, False, inv, True) - ref).max() <= 1e-9 * np.abs(ref).max()


def test_twiddle_tables_fit_their_slots():
    for L in [2 ** k for k in range(1, 14)] + [3 * 2 ** k for k in range(5, 13)]:
        f, r = tw_size(L, False), tw_size(L, True)
        assert f <= 2 * L and r <= 2 * L                 # FBP / Paganin: forward at 0, reversed at 2L
        if L <= 3072:
            assert f <= 3 * L // 2 and r <= 3 * L // 2  # propagator: forward at 0, reversed at 3L/2, 3L slot
    for L in (6144, 12288):
        assert tw_size(L, False, True) <= 2 * L          # Radon handle: 2L entries (4n)
