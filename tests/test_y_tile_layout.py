"""The y-pass's column tile (ibpm.jl_b200/csrc/dst_kernels.cuh, dst_y_kernel),
checked on the CPU for every transform length the library instantiates, both
scalar types and both plans.  `tests/y_tile_dump.cu` prints the tile
parameters from the header's own constexpr helpers (the functions the kernel
indexes with); this file restates them and checks:

* the restatement agrees with the header;
* element (row j, column c) at c·CS + off(j), off(j) = j + ⌊j/PI⌋, is
  one-to-one and stays inside the tile region the launch allocates, so no
  access reaches the FFT buffers placed after it;
* the post-processing scan's writes (thread t of a group emits outputs
  2(tC + s) and 2(tC + s) − 1) take at most 1.25× the ideal wavefronts over
  a transform, and no access more than 2×; the row-major fill and store (TW
  columns per row, consecutive threads) are free of bank conflicts;
* the transform's loads (consecutive rows of one column, ascending and
  descending) and the divide's are at most 2-way.

Bank model: 32 banks of 4 bytes.  A warp's 4-byte access takes as many
wavefronts as the largest number of distinct words in one bank; an 8-byte
access is served per half-warp, by 8-byte bank pairs."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ibpm.jl_b200", "csrc")


def lengths():
    src = open(os.path.join(ROOT, "ibpm.jl_b200", "csrc", "dst.cu")).read()
    m = re.search(r"#define IBPM_DST_LENGTHS\(X\)(.*)", src)
    return [int(x) for x in re.findall(r"X\((\d+)\)", m.group(1))]


# Plan helpers (dst_kernels.cuh: ct_fine, ct_tp, ct_groups, y_groups).
def ct_fine(N, PL):
    return N < 1024 and PL == 0


def ct_tp(N, PL):
    t = (((N // 4 if ct_fine(N, PL) else N // 8) + 31) // 32) * 32
    return max(t, 32)


def ct_groups(N, PL):
    tp = ct_tp(N, PL)
    return 1 if tp >= 128 else 128 // tp


def y_groups(N, esize, PL):
    if esize == 8 and ct_fine(N, PL) and ct_groups(N, PL) < 2:
        return 2
    return ct_groups(N, PL)


def round4(n):
    return ((n + 3) // 4) * 4


def c_mod(a, b):
    """C++ remainder (truncating toward zero)."""
    r = abs(a) % abs(b)
    return -r if a < 0 else r


def scan_run(N, PL):
    return (N // 2 + ct_tp(N, PL) - 1) // ct_tp(N, PL)


def pad_every(N, esize, PL):
    c = scan_run(N, PL)
    while c % 2 == 0:
        c //= 2
    return (128 // esize) * c


def col_stride(N, esize, PL, n2):
    E = 128 // esize
    TW = 2 * y_groups(N, esize, PL)
    R = E // TW if E // TW > 0 else 1
    PI = pad_every(N, esize, PL)
    base = (n2 - 1) + (n2 - 1) // PI + 2
    return base + c_mod(c_mod(R - c_mod(base, E), E) + E, E)


def tile_elems(N, esize, PL, n2):
    return round4(2 * y_groups(N, esize, PL) * col_stride(N, esize, PL, n2))


class Tile:
    """The layout as restated here, or (`dump`) as the header computes it."""

    def __init__(self, N, esize, PL, dump=None):
        self.N, self.esize, self.PL = N, esize, PL
        self.n2 = N - 1
        self.E = 128 // esize
        self.G = y_groups(N, esize, PL)
        self.TW = 2 * self.G
        self.TP = ct_tp(N, PL)
        self.run = scan_run(N, PL)
        self.PI = pad_every(N, esize, PL)
        self.CS = col_stride(N, esize, PL, N - 1)
        self.elems = tile_elems(N, esize, PL, self.n2)
        self.offs = [j + j // self.PI for j in range(self.n2)]
        if dump is not None:
            self.TW, self.TP, self.run, self.PI, self.CS, self.elems = dump["params"]
            self.offs = dump["offs"]

    def off(self, j):
        return self.offs[j]

    def at(self, j, c):
        return c * self.CS + self.off(j)

    def wavefronts(self, elems):
        """Wavefronts of one warp access to the given element indices (None =
        inactive lane)."""
        act = [e for e in elems if e is not None]
        if not act:
            return 0
        if self.esize == 4:
            return max_per_bank(act, lambda e: e % 32)
        total = 0
        for h in (elems[:16], elems[16:]):
            a = [e for e in h if e is not None]
            if a:
                total += max_per_bank(a, lambda e: e % 16)
        return total

    def ideal(self, elems):
        act = [e for e in elems if e is not None]
        if not act:
            return 0
        if self.esize == 4:
            return 1
        return sum(1 for h in (elems[:16], elems[16:]) if any(e is not None for e in h))


def max_per_bank(elems, bank):
    per = {}
    for e in set(elems):
        per.setdefault(bank(e), set()).add(e)
    return max(len(v) for v in per.values())


CONFIGS = [(N, es, PL) for N in lengths() for es in (4, 8) for PL in (0, 1)]


def cfg_id(c):
    return f"N{c[0]}-{'f64' if c[1] == 8 else 'f32'}-PL{c[2]}"


@pytest.fixture(scope="module")
def header_tiles(tmp_path_factory):
    """The header's tile parameters for every configuration, from
    tests/y_tile_dump.cu compiled for the host."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    exe = str(tmp_path_factory.mktemp("ytile") / "y_tile_dump")
    subprocess.run([nvcc, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a", "-I", CSRC,
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "y_tile_dump.cu"), "-o", exe],
                   check=True, capture_output=True, timeout=300)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=60).stdout
    tiles = {}
    for line in out.splitlines():
        v = [int(x) for x in line.split()]
        N, es, PL = v[:3]
        tiles[(N, es, PL)] = {"params": tuple(v[3:9]), "offs": v[9:]}
    return tiles


def test_dump_covers_every_length(header_tiles):
    assert sorted(header_tiles) == sorted(CONFIGS)


@pytest.mark.parametrize("cfg", CONFIGS, ids=cfg_id)
def test_restatement_agrees_with_the_header(cfg, header_tiles):
    mine, theirs = Tile(*cfg), Tile(*cfg, dump=header_tiles[cfg])
    assert (mine.TW, mine.TP, mine.run, mine.PI, mine.CS, mine.elems) == \
        (theirs.TW, theirs.TP, theirs.run, theirs.PI, theirs.CS, theirs.elems)
    assert mine.offs == theirs.offs


@pytest.mark.parametrize("cfg", CONFIGS, ids=cfg_id)
def test_tile_is_one_to_one_and_in_bounds(cfg, header_tiles):
    t = Tile(*cfg, dump=header_tiles[cfg])
    seen = set()
    for c in range(t.TW):
        for j in range(t.n2):
            a = t.at(j, c)
            assert 0 <= a < t.elems, (j, c, a, t.elems)
            seen.add(a)
    assert len(seen) == t.TW * t.n2
    # the columns of the group's pair never overlap: one column fits its stride
    assert t.off(t.n2 - 1) < t.CS
    # at most 15% more shared memory than the row-major tile of pitch TW + 1
    assert t.elems <= 1.15 * round4(t.n2 * (t.TW + 1)) + 4 * t.E


def scan_cost(t, off):
    """(wavefronts, ideal wavefronts, worst access ratio) of the scan's writes
    to one column over a transform."""
    half = t.N // 2
    C = (half + t.TP - 1) // t.TP
    tot = ideal = 0
    worst = 0.0
    for warp in range(t.TP // 32):
        for s in range(C):
            for odd in (0, 1):
                elems = []
                for lane in range(32):
                    k = (warp * 32 + lane) * C + s
                    o = 2 * k - odd
                    ok = k < half and (odd == 0 or k > 0)
                    elems.append(off(o) if ok else None)
                w, i = t.wavefronts(elems), t.ideal(elems)
                tot += w
                ideal += i
                if i:
                    worst = max(worst, w / i)
    return tot, ideal, worst


@pytest.mark.parametrize("cfg", CONFIGS, ids=cfg_id)
def test_scan_emits_are_near_conflict_free(cfg, header_tiles):
    t = Tile(*cfg, dump=header_tiles[cfg])
    tot, ideal, worst = scan_cost(t, t.off)
    assert tot <= 1.25 * ideal and worst <= 2.0, (tot, ideal, worst)


@pytest.mark.parametrize("cfg", CONFIGS, ids=cfg_id)
def test_row_major_fill_and_store_are_free_of_bank_conflicts(cfg, header_tiles):
    t = Tile(*cfg, dump=header_tiles[cfg])
    total = t.n2 * t.TW
    for base in range(0, total, 32):
        elems = []
        for lane in range(32):
            idx = base + lane
            elems.append(t.at(idx // t.TW, idx % t.TW) if idx < total else None)
        assert t.wavefronts(elems) == t.ideal(elems), base


@pytest.mark.parametrize("cfg", CONFIGS, ids=cfg_id)
def test_transform_loads_are_at_most_two_way(cfg, header_tiles):
    t = Tile(*cfg, dump=header_tiles[cfg])
    half = t.N // 2
    IT = (half + t.TP) // t.TP
    for warp in range(t.TP // 32):
        for it in range(IT):
            up, down = [], []
            for lane in range(32):
                m = warp * 32 + lane + it * t.TP
                up.append(t.off(m - 1) if 1 <= m <= half else None)
                down.append(t.off(t.N - m - 1) if 1 <= m < half else None)
            for elems in (up, down):
                assert t.wavefronts(elems) <= 2 * t.ideal(elems)
    # the divide: o = tid + k·TP
    for warp in range(t.TP // 32):
        for k in range((t.n2 + t.TP - 1) // t.TP):
            elems = [t.off(o) if o < t.n2 else None
                     for o in (warp * 32 + lane + k * t.TP for lane in range(32))]
            assert t.wavefronts(elems) <= 2 * t.ideal(elems)


def test_the_layouts_it_replaced_had_the_scan_conflicts():
    """The row-major tile of pitch TW + 1 took 8x the ideal wavefronts for the
    scan of the FP64 throughput plan at N = 512; a pad every line (whatever
    the run length) took 3.5x at N = 192, where each thread's run is 3."""
    t = Tile(512, 8, 1)
    tot, ideal, _ = scan_cost(t, lambda o: o * (t.TW + 1))
    assert tot >= 8 * ideal
    t = Tile(192, 8, 1)
    assert t.run == 3
    tot, ideal, _ = scan_cost(t, lambda o: o + o // t.E)
    assert tot >= 3 * ideal
    tot, ideal, _ = scan_cost(t, t.off)
    assert tot <= 1.1 * ideal
