"""CPU restatement of the 16 x 256 split 4096-point kernel's index maps
(fft_tma_split_kernel in aocl-fftz_b200/csrc/kernels/fft_tma.cu), checked
without a GPU:

* the TMA staging image (box s = elements [256 s, 256 s + 256) of the tile's
  four transforms, [n0][m_l][col] with the 32-byte swizzle for column tiles,
  [row][m_l][n0] with the 128-byte swizzle for row tiles) and the stage-a read
  offset rd0 of every lane: it picks x[p][n0 + 16 (l + 16 s)];
* the transpose slots inside each warp's own staging slice (offset
  l * 1024 + wb + (u ^ f(k)) written, x * 1024 + wb + (u ^ f(x)) read): a
  bijection onto the slice;
* both exchange layouts (full complex, two k' rounds; one real component);
* every shared-memory instruction conflict-free per half-warp (16 distinct
  8-byte bank pairs) or per warp (32 distinct 4-byte banks);
* the whole tile computed through these maps equals numpy's FFT.
"""
import numpy as np
import pytest

N = 4096


def lane_gl(lane):
    return (lane >> 3) & 1, (lane & 7) | ((lane >> 4) << 3)


def split_f(mode, d):
    if mode == 1:
        return ((d & 7) << 2) | (((d >> 2) & 1) << 1) | ((d >> 3) & 1)
    return ((d & 7) << 4) | ((d & 7) << 1) | ((d >> 3) & 1)


def warp_consts(mode, w, g, l):
    """pw, n0w, wb, u, rd0 as the kernel computes them."""
    if mode == 1:
        a = w & 1
        n0w, pw, wb = w >> 1, 2 * a + g, (w >> 1) * 64
        c = (33 * g) ^ (2 * a)
        rd0 = wb + ((l * 4 + 2 * ((l >> 2) & 1) + g) ^ (2 * a))
    else:
        b = w & 7
        pw, n0w, wb = w >> 3, 2 * b + g, (w >> 3) * 256
        c = (129 * g) ^ (2 * b)
        rd0 = wb + ((l * 16 + 2 * (l & 7) + g) ^ (2 * b))
    return pw, n0w, wb, split_f(mode, l) ^ c, rd0


def staged_image(mode, x):
    img = np.zeros(16384, np.complex128)
    seen = np.zeros(16384, int)
    for s in range(16):
        for m_l in range(16):
            for n0 in range(16):
                for p in range(4):
                    if mode == 1:  # byte n0*512 + m_l*32 + p*8, bit 4 ^= bit 7
                        idx = s * 1024 + n0 * 64 + m_l * 4 + (p ^ (((m_l >> 2) & 1) << 1))
                    else:  # byte p*2048 + m_l*128 + n0*8, bits 4-6 ^= bits 7-9
                        idx = s * 1024 + p * 256 + m_l * 16 + (((n0 >> 1) ^ (m_l & 7)) << 1) + (n0 & 1)
                    img[idx] = x[p][n0 + 16 * (m_l + 16 * s)]
                    seen[idx] += 1
    assert (seen == 1).all()
    return img


def conflict_free_64(addrs):
    for h in range(2):
        assert len({a % 16 for a in addrs[16 * h:16 * h + 16]}) == 16


def conflict_free_32(addrs):
    assert len({a % 32 for a in addrs}) == 32


def reader(omode, t):
    return (t & 3, t >> 2) if omode == 1 else (t >> 8, t & 255)


def exch_complex(p, n0, kl):
    return (p * 16 + n0) * 128 + (kl ^ (4 * ((p >> 1) & 1) + 8 * ((p ^ n0) & 1)))


def exch_real(p, n0, kp):
    return (p * 16 + n0) * 256 + (kp ^ (8 * ((p >> 1) & 1) + 16 * ((p ^ n0) & 1)))


def run_tile(mode, omode, xm, x):
    W256 = np.exp(-2j * np.pi * np.arange(256) / 256)
    W4096 = np.exp(-2j * np.pi * np.arange(4096) / 4096)
    img = staged_image(mode, x)
    z = {}
    for w in range(32):
        consts = [warp_consts(mode, w, *lane_gl(ln)) for ln in range(32)]
        slice_set = set()
        for ln in range(32):
            g, l = lane_gl(ln)
            pw, n0w, wb, u, rd0 = consts[ln]
            for s in range(16):
                slice_set.add(s * 1024 + rd0)
                assert img[s * 1024 + rd0] == x[pw][n0w + 16 * (l + 16 * s)]
        assert len(slice_set) == 512
        for s in range(16):
            conflict_free_64([s * 1024 + c[4] for c in consts])
        v = {}
        for ln in range(32):
            g, l = lane_gl(ln)
            vv = np.fft.fft(np.array([img[s * 1024 + consts[ln][4]] for s in range(16)]))
            v[ln] = vv * W256[(l * np.arange(16)) % 256]
        mem = {}
        for k in range(16):
            addrs = []
            for ln in range(32):
                g, l = lane_gl(ln)
                a = l * 1024 + consts[ln][2] + (consts[ln][3] ^ split_f(mode, k))
                assert a in slice_set and a not in mem
                mem[a] = v[ln][k]
                addrs.append(a)
            conflict_free_64(addrs)
        assert set(mem) == slice_set
        for xx in range(16):
            conflict_free_64([xx * 1024 + c[2] + (c[3] ^ split_f(mode, xx)) for c in consts])
        for ln in range(32):
            g, l = lane_gl(ln)
            pw, n0w, wb, u, rd0 = consts[ln]
            vals = np.array([mem[xx * 1024 + wb + (u ^ split_f(mode, xx))] for xx in range(16)])
            z[(pw, n0w, l)] = np.fft.fft(vals)  # Z_n0[l + 16 k_hi]
    # exchange: gather Z_n0[k'] for reader (p, k')
    X = {}
    if xm == 1:
        for rnd in range(2):
            for w in range(32):
                for kh in range(8):
                    addrs = []
                    for ln in range(32):
                        g, l = lane_gl(ln)
                        pw, n0w = warp_consts(mode, w, g, l)[:2]
                        a = exch_complex(pw, n0w, l + 16 * kh)
                        assert (rnd, a) not in X
                        X[(rnd, a)] = z[(pw, n0w, l)][8 * rnd + kh]
                        addrs.append(a)
                    conflict_free_64(addrs)
            assert sorted(a for r, a in X if r == rnd) == list(range(8192))
            for w in range(32):
                if (reader(omode, 32 * w)[1] >> 7) != rnd:
                    continue
                for n0 in range(16):
                    conflict_free_64([exch_complex(*reader(omode, 32 * w + ln)[:1], n0,
                                                   reader(omode, 32 * w + ln)[1] & 127) for ln in range(32)])
    else:
        for part in range(2):
            for w in range(32):
                for kh in range(16):
                    addrs = []
                    for ln in range(32):
                        g, l = lane_gl(ln)
                        pw, n0w = warp_consts(mode, w, g, l)[:2]
                        a = exch_real(pw, n0w, l + 16 * kh)
                        X[(part, a)] = z[(pw, n0w, l)][kh]
                        addrs.append(a)
                    conflict_free_32(addrs)
            assert sorted(a for r, a in X if r == part) == list(range(16384))
            for w in range(32):
                for n0 in range(16):
                    conflict_free_32([exch_real(reader(omode, 32 * w + ln)[0], n0, reader(omode, 32 * w + ln)[1])
                                      for ln in range(32)])
    out = np.zeros((4, N), np.complex128)
    for t in range(1024):
        p, kp = reader(omode, t)
        if xm == 1:
            vals = np.array([X[(kp >> 7, exch_complex(p, n0, kp & 127))] for n0 in range(16)])
        else:
            vals = np.array([X[(0, exch_real(p, n0, kp))] for n0 in range(16)])
        y = np.fft.fft(vals * W4096[(np.arange(16) * kp) % 4096])
        out[p][kp + 256 * np.arange(16)] = y
    return out


@pytest.mark.parametrize("mode", [1, 0])
@pytest.mark.parametrize("omode", [1, 0])
@pytest.mark.parametrize("xm", [0, 1])
def test_split_tile_maps(mode, omode, xm):
    rng = np.random.default_rng(10 * mode + 2 * omode + xm)
    x = rng.standard_normal((4, N)) + 1j * rng.standard_normal((4, N))
    y = run_tile(mode, omode, xm, x)
    ref = np.fft.fft(x, axis=1)
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-12


def test_one_component_writer_bases():
    """The kernel writes value k_hi at (k_hi odd ? xfw_o : xfw_e) + 16 k_hi."""
    for mode in (1, 0):
        for w in range(32):
            for ln in range(32):
                g, l = lane_gl(ln)
                pw, n0w = warp_consts(mode, w, g, l)[:2]
                sw1 = 8 * ((pw >> 1) & 1) + 16 * ((pw ^ n0w) & 1)
                xfw = (pw * 16 + n0w) * 256 + (l ^ (sw1 & 15))
                s4 = 16 * (sw1 >> 4)
                for kh in range(16):
                    assert exch_real(pw, n0w, l + 16 * kh) == ((xfw - s4) if kh & 1 else (xfw + s4)) + 16 * kh


def test_blocked_intermediate_addresses_agree():
    """The 4096 x 4096 four-step's blocked intermediate: the column pass
    stores output k1 of column j2 at obase + jo + 256 r * oes (rr_store,
    k1 = j + 256 r, obase = line * n + j2, jo = (j >> 2) 4 oes + (j & 3) + 3 j2),
    the row pass's tensor map reads element e of row k1 = 4 K + rr through
    dims (rr, m, n0, K) with strides (1, 64, 4, 4 n2) elements (e = n0 + 16 m);
    both must be the same bijection onto [0, n)."""
    n1 = n2 = 4096
    oes = n2
    j2 = np.arange(n2)[:, None]
    k1 = np.arange(n1)[None, :]
    j, r = k1 % 256, k1 // 256
    store = (j2 + (j >> 2) * 4 * oes + (j & 3) + 3 * j2) + 256 * r * oes
    K, rr = k1 // 4, k1 % 4
    e = j2
    n0, m = e % 16, e // 16
    load = rr * 1 + m * 64 + n0 * 4 + K * 4 * n2
    assert (store == load).all()
    assert len(np.unique(store)) == n1 * n2 and store.min() == 0 and store.max() == n1 * n2 - 1
