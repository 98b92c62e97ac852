"""Seeded synthetic slot generator (the project's own; numpy, host side).

No public dataset is involved: the reference generates its vectors with a
MATLAB script (matlab/data_generator.m), and the workloads here are seeded
synthetic slots with the shapes and statistics of the configurations this
build is measured on.  A slot holds P comb-pilot symbols followed by U
uplink data symbols, each an [M][N] array of time-domain antenna samples.

Pilots follow the reference's comb layout (fft_callback.cuh:76-108): on pilot
symbol p, subcarrier i carries user p*sg + (i % sg) with the value
p_raw[i], where p_raw / |p_raw|^2 is the receiver's pilot table
(fft_op.cu:176-192).  Data bits are scrambled, mapped with the Gray tables
that the reference's soft demapper inverts (modulation/demodulation.h:30-67;
for 256-QAM the reference's table is inverted on every bit relative to its
demapper, so the generator flips the index to stay consistent), and placed
on subcarrier s as stream bits s*Qm .. s*Qm+Qm-1.

Channels: "iid_group" draws CN(0,1) per (group of sg subcarriers, antenna,
user); "tdl" draws an n_taps exponential power-delay-profile channel with
exponential antenna correlation rho (Kronecker, receive side), normalised
to unit average power per link; "tdl_ds" is the same with the taps spread
over three delay spreads given in nanoseconds (tap_profile).  AWGN is added per subcarrier at the stated
per-user SNR.
"""
from dataclasses import dataclass, field

import numpy as np

# The generator is plain numpy and imports nothing else from this package, so
# that a process which must not load the library (a timing run of the
# reference's own operators) can still build the same seeded slots.


@dataclass
class CellConfig:
    M: int = 64            # antennas
    K: int = 16            # users
    N: int = 2048          # FFT size
    S: int = 1200          # data subcarriers
    sg: int = 16           # subcarrier group
    Qm: int = 4            # bits per QAM symbol
    U: int = 13            # uplink data symbols per slot
    snr_db: float = 20.0
    channel: str = "iid_group"   # or "tdl", "tdl_ds"
    n_taps: int = 8
    tap_decay: float = 2.0       # PDP e^{-l / tap_decay}, in samples
    rho: float = 0.0             # antenna correlation
    delay_spread_ns: float = 0.0  # tdl_ds: exponential PDP decay constant
    scs_hz: float = 30e3          # subcarrier spacing (tdl_ds)
    iq_dtype: str = "c64"        # c64 | int16 | int8 | f16
    scrambler: str = "lfsr127"   # lfsr127 | gold
    c_init: int = 0x1234
    code_rate: float = 1.0 / 3.0
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def P(self):
        return (self.K + self.sg - 1) // self.sg  # config.cc:75-82, main.cc:67

    @property
    def G(self):
        return (self.S + self.sg - 1) // self.sg

    @property
    def start(self):
        return (self.N - self.S) // 2  # config.cc:31

    @property
    def symbols(self):
        return self.P + self.U

    def ldpc(self):
        """(cb_size, zeros, cb_stride): encoded bits, punctured bits and the
        tight row stride of the LLR layout for one code block per symbol."""
        e, p, _ = ldpc_sizes(self.S, self.Qm, self.code_rate)
        return e, p, e + p


# TS 38.212 Table 5.3.2-1 lifting sizes, ascending
_LIFTING = sorted([2, 4, 8, 16, 32, 64, 128, 256, 3, 6, 12, 24, 48, 96, 192, 384, 5, 10, 20, 40, 80, 160,
                   320, 7, 14, 28, 56, 112, 224, 9, 18, 36, 72, 144, 288, 11, 22, 44, 88, 176, 352, 13, 26,
                   52, 104, 208, 15, 30, 60, 120, 240])


def ldpc_sizes(S, Qm, code_rate=1.0 / 3.0, base_graph=1, pilot_spacing=0, downlink=False):
    """(encoded, punctured, decoded) bits of one code block, the sizing of
    config/config.cc:84-135: the largest lifting size Zc with kb*Zc not above
    the symbol's uncoded bits (kb = 22 for BG1, 10 for BG2), round(kb/rate)
    - (kb-2) parity rows, the first 2*Zc systematic bits punctured.  Host
    arithmetic, the same as the library's mb_ldpc_sizes."""
    kb = 22 if base_graph == 1 else 10
    data = S - S // pilot_spacing if (downlink and pilot_spacing) else S
    uncoded = int(float(data * Qm) * code_rate)
    z = _LIFTING[-1]
    for a, b in zip(_LIFTING[:-1], _LIFTING[1:]):
        if kb * a <= uncoded < kb * b:
            z = a
            break
    rows = int(np.floor(kb / code_rate + 0.5)) - (kb - 2)
    return (kb - 2 + rows) * z, 2 * z, kb * z


def _zc_length(S):
    """utils.h:56-62: the largest prime <= S from the table ending at 2039,
    2039 itself when S is larger or nothing matches."""
    n = 2039
    sieve = np.ones(n + 1, bool)
    sieve[:2] = False
    for d in range(2, int(n ** 0.5) + 1):
        if sieve[d]:
            sieve[d * d::d] = False
    primes = np.nonzero(sieve[:min(S, n) + 1])[0]
    return 2039 if (len(primes) == 0 or S >= 2039) else int(primes[-1])


def pilot_values(S):
    """The transmitted comb pilot of subcarrier i, p[i] = zc(i mod L) e^{j pi i / 4}
    (fft/fft_op.cu:176-192 over utils.h:54-95; the receiver's table is
    p / |p|^2): Zadoff-Chu of length L, the largest prime <= S, root
    round(2L/31), phases rounded to float as the reference forms them."""
    L = _zc_length(S)
    root = np.floor(L * 2.0 / 31.0 + 0.5)
    i = np.arange(S, dtype=np.int64)
    m = (i % L).astype(np.float64)
    th = (-np.pi * root * m * (m + 1) / L).astype(np.float32).astype(np.float64)
    a = (np.float32(np.pi / 4) * i.astype(np.float32)).astype(np.float64)
    return np.exp(1j * (th + a)).astype(np.complex64)


def mod_table(Qm):
    """Reference Gray tables (modulation.cu:22-72)."""
    if Qm == 2:
        s = np.float32(1 / np.sqrt(2))
        v = np.array([-s, s], np.float32)
        idx = np.arange(4)
        return (v[idx // 2] + 1j * v[idx % 2]).astype(np.complex64)
    if Qm == 4:
        s = np.float32(1 / np.sqrt(10))
        v = np.array([1, 3, -1, -3], np.float32) * s
        i = np.arange(16)
        im = (((i >> 2) & 1) << 1) + (i & 1)
        re = (((i >> 3) & 1) << 1) + ((i >> 1) & 1)
        return (v[re] + 1j * v[im]).astype(np.complex64)
    if Qm == 6:
        s = np.float32(1 / np.sqrt(42))
        v = np.array([3, 1, 5, 7, -3, -1, -5, -7], np.float32) * s
        i = np.arange(64)
        im = (((i >> 4) & 1) << 2) + (((i >> 2) & 1) << 1) + (i & 1)
        re = (((i >> 5) & 1) << 2) + (((i >> 3) & 1) << 1) + ((i >> 1) & 1)
        return (v[re] + 1j * v[im]).astype(np.complex64)
    s = np.float32(1 / np.sqrt(170))
    v = np.array([-15, -13, -9, -11, -1, -3, -7, -5, 15, 13, 9, 11, 1, 3, 7, 5], np.float32) * s
    i = np.arange(256)
    im = ((i & 0x40) >> 3) + ((i & 0x10) >> 2) + ((i & 0x4) >> 1) + (i & 0x1)
    re = ((i & 0x80) >> 4) + ((i & 0x20) >> 3) + ((i & 0x8) >> 2) + ((i & 0x2) >> 1)
    return (v[re] + 1j * v[im]).astype(np.complex64)


def lfsr127():
    """scrambler.cu:22-31."""
    s, out = 0x5D, np.zeros(127, np.uint8)
    for i in range(127):
        fb = (s ^ (s >> 3)) & 1
        out[i] = fb
        s = (s >> 1) | (fb << 6)
    return out


def gold(c_init, n):
    """TS 38.211 5.2.1 Gold sequence c(0..n-1)."""
    Nc = 1600
    x1 = np.zeros(n + Nc + 31, np.uint8)
    x2 = np.zeros(n + Nc + 31, np.uint8)
    x1[0] = 1
    x2[:31] = [(c_init >> i) & 1 for i in range(31)]
    for k in range(n + Nc):
        x1[k + 31] = x1[k + 3] ^ x1[k]
        x2[k + 31] = x2[k + 3] ^ x2[k + 2] ^ x2[k + 1] ^ x2[k]
    return x1[Nc:Nc + n] ^ x2[Nc:Nc + n]


def scrambling_bits(cfg, n_bits):
    """[K][n_bits] descrambling sequence per user, as the receiver uses it."""
    if cfg.scrambler == "gold":
        return np.stack([gold(cfg.c_init + u, n_bits) for u in range(cfg.K)])
    seq = lfsr127()
    return np.tile(seq[np.arange(n_bits) % 127], (cfg.K, 1))


def tap_profile(cfg):
    """Tap delays (in samples) and powers of the TDL channels.  "tdl": taps at
    0..L-1 samples with PDP e^{-l / tap_decay}.  "tdl_ds": L taps spread over
    [0, 3 ds] with PDP e^{-tau / ds}, ds = delay_spread_ns at the sample rate
    N * scs_hz (fractional delays)."""
    L = cfg.n_taps
    if cfg.channel == "tdl_ds":
        fs = cfg.N * cfg.scs_hz
        ds = max(cfg.delay_spread_ns, 1e-3) * 1e-9 * fs
        tau = np.arange(L) * (3.0 * ds / max(L - 1, 1))
        pdp = np.exp(-tau / ds)
    else:
        tau = np.arange(L, dtype=np.float64)
        pdp = np.exp(-tau / cfg.tap_decay)
    return tau, pdp / pdp.sum()


def _channel(cfg, rng):
    """Frequency response H[s][b][u] (complex64) on the S data subcarriers."""
    M, K, S, sg = cfg.M, cfg.K, cfg.S, cfg.sg
    if cfg.channel == "iid_group":
        G = cfg.G
        h = (rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K))) / np.sqrt(2)
        return h[np.arange(S) // sg].astype(np.complex64)
    # tdl: taps[l][b][u] with exponential PDP and receive correlation
    L = cfg.n_taps
    tau, pdp = tap_profile(cfg)
    w = (rng.standard_normal((L, M, K)) + 1j * rng.standard_normal((L, M, K))) / np.sqrt(2)
    if cfg.rho:
        idx = np.arange(M)
        R = cfg.rho ** np.abs(idx[:, None] - idx[None, :])
        Rh = np.linalg.cholesky(R)
        w = np.einsum("ab,lbk->lak", Rh, w)
    taps = w * np.sqrt(pdp)[:, None, None]
    bins = (np.arange(S) + cfg.start + cfg.N // 2) % cfg.N
    # the data bins' physical frequency offset relative to DC
    f = ((bins + cfg.N // 2) % cfg.N) - cfg.N // 2
    ph = np.exp(-2j * np.pi * np.outer(f, tau) / cfg.N)  # [S][L], tau in samples
    H = np.tensordot(ph, taps, axes=(1, 0))  # [S][M][K]
    return H.astype(np.complex64)


def _to_time(cfg, Y, gain):
    """Y [sym][M][S] frequency samples -> [sym][M][N] time samples (numpy
    inverse FFT, so the receiver's unnormalised forward FFT returns Y*gain)."""
    n_sym = Y.shape[0]
    row = np.zeros((n_sym, cfg.M, cfg.N), np.complex64)
    bins = (np.arange(cfg.S) + cfg.start + cfg.N // 2) % cfg.N
    row[:, :, bins] = Y * gain
    x = np.fft.ifft(row, axis=-1).astype(np.complex64)
    if cfg.iq_dtype == "c64":
        return x
    iq = np.stack([x.real, x.imag], axis=-1)
    if cfg.iq_dtype == "f16":
        return iq.astype(np.float16)
    qmax = 32767 if cfg.iq_dtype == "int16" else 127
    q = np.clip(np.rint(iq * (qmax + 1)), -qmax - 1, qmax)
    return q.astype(np.int16 if cfg.iq_dtype == "int16" else np.int8)


def make_slot(cfg, coded=None):
    """Returns a dict: iq [P+U][M][N](...), H [S][M][K], bits [U][K][S*Qm]
    (transmitted coded bits, before scrambling), x [U][K][S] (transmitted
    QAM symbols), noise_var, pilot_raw [S], seq [K][S*Qm].  With coded
    ([U][K][S*Qm] 0/1, e.g. LDPC codewords of scrambled information bits,
    the reference's order, process.cc:196-214) those bits are sent as they
    are: no scrambling of the coded bits."""
    rng = np.random.default_rng(np.random.Philox(cfg.seed))
    M, K, S, sg, Qm, U, P = cfg.M, cfg.K, cfg.S, cfg.sg, cfg.Qm, cfg.U, cfg.P
    H = _channel(cfg, rng)
    pilot_raw = pilot_values(S)
    nbits = S * Qm
    bits = rng.integers(0, 2, (U, K, nbits), dtype=np.uint8)
    seq = scrambling_bits(cfg, nbits)
    tx = bits ^ seq[None]
    if coded is not None:
        bits = tx = np.asarray(coded, np.uint8).reshape(U, K, nbits)
    weights = 1 << np.arange(Qm - 1, -1, -1)
    idx = (tx.reshape(U, K, S, Qm) * weights).sum(-1)
    if Qm == 8:
        idx = idx ^ 0xFF
    X = mod_table(Qm)[idx]  # [U][K][S]
    noise_var = 10.0 ** (-cfg.snr_db / 10.0)

    Yp = np.zeros((P, M, S), np.complex64)
    s_idx = np.arange(S)
    for p in range(P):
        users = p * sg + (s_idx % sg)
        ok = users < K
        # H[s][:, users[s]] * pilot[s]
        hs = H[s_idx[ok], :, users[ok]]  # [n_ok][M]
        Yp[p][:, s_idx[ok]] = (hs * pilot_raw[s_idx[ok], None]).T
    Yu = np.matmul(H[None], X.transpose(0, 2, 1)[..., None])[..., 0]  # [U][S][M]
    Yu = Yu.transpose(0, 2, 1)
    Y = np.concatenate([Yp, Yu]).astype(np.complex64)
    nz = (rng.standard_normal(Y.shape) + 1j * rng.standard_normal(Y.shape)) * np.sqrt(noise_var / 2)
    Y = (Y + nz).astype(np.complex64)
    # the unnormalised FFT of numpy's ifft returns Y; int formats get a gain
    # that puts the time-domain RMS near a quarter of full scale
    gain = 1.0
    if cfg.iq_dtype in ("int16", "int8"):
        rms = np.sqrt(np.mean(np.abs(Y) ** 2) * S) / cfg.N
        gain = 0.25 / max(rms, 1e-12)
    iq = _to_time(cfg, Y, gain)
    return dict(iq=iq, H=H, bits=bits, x=X, noise_var=noise_var, pilot_raw=pilot_raw,
                seq=seq, gain=gain, Y=Y)


# data subcarriers and their FFT size, as the batched-cells workload pairs them
CELL_SUBCARRIERS = {600: 1024, 1200: 2048, 3276: 4096}


def make_cells(n=32, seed=3, symbols=14, sg=16, snr_db=(15.0, 25.0), M_set=(32, 64, 128),
               K_set=(4, 8, 16, 32), S_set=(600, 1200, 3276), Qm_set=(2, 4, 6)):
    """Seeded configurations of n uneven cells: antennas from M_set, users
    from K_set (K <= M), data subcarriers from S_set with the FFT size of
    CELL_SUBCARRIERS, QAM order from Qm_set, i.i.d. Rayleigh channels per
    subcarrier group, per-cell SNR uniform in snr_db; P = ceil(K / sg) comb
    pilot symbols and U = symbols - P data symbols."""
    rng = np.random.default_rng(seed)
    cfgs = []
    for c in range(n):
        M = int(rng.choice(M_set))
        K = int(rng.choice([k for k in K_set if k <= M]))
        S = int(rng.choice(S_set))
        Qm = int(rng.choice(Qm_set))
        P = (K + sg - 1) // sg
        cfgs.append(CellConfig(M=M, K=K, N=CELL_SUBCARRIERS[S], S=S, sg=sg, Qm=Qm, U=symbols - P,
                               snr_db=float(rng.uniform(*snr_db)), channel="iid_group",
                               seed=int(rng.integers(1 << 31))))
    return cfgs
