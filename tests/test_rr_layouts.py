"""Shared-memory index arithmetic of the register-resident 4096-point kernel
(fft_tma_rr_kernel in aocl-fftz_b200/csrc/kernels/fft_tma.cu), restated and
checked on the CPU for every thread and every value of a tile of four
transforms (1024 threads, 16 values a thread):

* each exchange writes every slot of its layout exactly once and the next
  stage reads exactly those slots back, in bounds of the buffer;
* every warp-wide access of one value index r touches 32 distinct banks with
  distinct words (no bank conflict), for both lane maps (rows: one transform
  per warp; columns: four transforms per warp);
* the value each reader gets is the one the right writer stored (the
  exchange implements the Stockham stage permutation);
* the CTA's shared memory fits the 196 KB carveout."""
import pytest

N, TPC, TPT, R = 4096, 4, 256, 16
SSF1, SH1 = 4228, 5  # exchange 1: one pad word per 32, transforms 4228 words apart


def lane(mode, t):
    return (t // TPT, t % TPT) if mode == 0 else (t % TPC, t // TPC)


def phys(i, sh):
    return i + (i >> sh)


def ex1_write(p, j, r):  # stage 0 outputs (Ns = 1): element 16 j + r
    return p * SSF1 + phys(16 * j + r, SH1)


def ex1_read(p, j, r):  # stage 1 inputs: element j + 256 r
    return p * SSF1 + phys(j + 256 * r, SH1)


def ex2_layout(p, i):
    return p * 4096 + (i ^ (((i >> 8) & 1) << 4) ^ (8 * p))


def ex2_write(p, j, r):  # two bases per thread, as rr_exchange_x computes them
    key = (((j >> 4) & 1) << 4) ^ (8 * p)
    kb = key >> 4 & 1
    wb = p * 4096 + ((((j >> 4) << 8) + (j & 15)) ^ (key & 8))
    return (wb - 16 * kb if r & 1 else wb + 16 * kb) + 16 * r


def ex2_read(p, j, r):
    re = p * 4096 + (j ^ (8 * p))
    return (re ^ 16 if r & 1 else re) + 256 * r


def conflict_free(addrs):
    banks = {}
    for a in addrs:
        banks.setdefault(a % 32, set()).add(a)
    return all(len(s) == 1 for s in banks.values()) and len(banks) == 32


@pytest.mark.parametrize("first_map", [1, 0])  # column pass (pass A) / row pass (pass B)
def test_exchange1(first_map):
    written = {}
    for t in range(TPC * TPT):
        p, j = lane(first_map, t)
        for r in range(R):
            a = ex1_write(p, j, r)
            assert 0 <= a < TPC * SSF1 and a not in written
            written[a] = (p, 16 * j + r)  # transform, stage-0 output index
    read = set()
    for t in range(TPC * TPT):
        p, j = lane(0, t)
        for r in range(R):
            a = ex1_read(p, j, r)
            assert written[a] == (p, j + 256 * r)
            read.add(a)
    assert read == set(written)
    for w in range(TPC * TPT // 32):
        for r in range(R):
            assert conflict_free([ex1_write(*lane(first_map, 32 * w + l), r) for l in range(32)])
            assert conflict_free([ex1_read(*lane(0, 32 * w + l), r) for l in range(32)])


@pytest.mark.parametrize("last_map", [1, 0])  # column (transposed or column store) / row store
def test_exchange2(last_map):
    written = {}
    for t in range(TPC * TPT):
        p, j = lane(0, t)
        k = j & 15
        d0 = (j - k) * 16 + k  # stage 1 (Ns = 16) outputs d0 + 16 r
        for r in range(R):
            a = ex2_write(p, j, r)
            assert a == ex2_layout(p, d0 + 16 * r)
            assert 0 <= a < TPC * 4096 and a not in written
            written[a] = (p, d0 + 16 * r)
    read = set()
    for t in range(TPC * TPT):
        p, j = lane(last_map, t)
        for r in range(R):
            a = ex2_read(p, j, r)
            assert a == ex2_layout(p, j + 256 * r)
            assert written[a] == (p, j + 256 * r)
            read.add(a)
    assert read == set(written)
    for w in range(TPC * TPT // 32):
        for r in range(R):
            assert conflict_free([ex2_write(*lane(0, 32 * w + l), r) for l in range(32)])
            assert conflict_free([ex2_read(*lane(last_map, 32 * w + l), r) for l in range(32)])


def test_exchange1_y_parts_fit_the_staging_area():
    # exchange 1's y parts use the consumed staged tile (4 x 4096 complex floats)
    assert TPC * SSF1 * 4 <= TPC * N * 8
    # exchange 2's y parts share the exchange buffer (x then y)
    assert TPC * 4096 <= TPC * SSF1


def test_shared_memory_fits_the_196kb_carveout():
    staged = TPC * N * 8          # staged tile, complex float
    xbuf = TPC * SSF1 * 4         # one-component exchange buffer
    offsets = 8 * TPC * 8         # two sets of {out, col} offsets and of the four-step steps
    dynamic = staged + xbuf + offsets + 128  # + alignment slack (the launcher's formula)
    assert dynamic + 1024 + 16 <= 196 * 1024  # + the block's reserved and static shared memory
