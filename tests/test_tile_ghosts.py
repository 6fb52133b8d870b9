"""The boundary unknowns ("ghosts") of the tiled smoother, checked on the CPU.

The tile kernels (imau-ice_b200/csrc/solver.cu, TileMem::ghosts_u / ghosts_v) keep every
boundary unknown of a tile equal to its source's value and rewrite it, by a direct rule,
when the source is updated.  The source is the boundary elimination's (solver.cu
u_src / v_src, the reference's boundary rows ice_velocity_module.f90:1932-2191).  These
tests restate both in Python and check, for every combination of 'zero' and 'infinite'
sides and several grid shapes, that (1) the direct rule writes exactly the boundary
unknowns whose source is the updated point, and (2) a row's outside same-component
neighbours map back to the row itself or to zero, so no colour pass reads a ghost that it
rewrites."""
import itertools

ZERO, INF, PER = 0, 1, 2
def pick(a, b):
    if a == ZERO or b == ZERO: return ZERO
    if a == INF or b == INF: return INF
    return PER
def u_int(nx, ny, j, i): return 1 <= i <= nx - 3 and 1 <= j <= ny - 2
def v_int(nx, ny, j, i): return 1 <= i <= nx - 2 and 1 <= j <= ny - 3
def u_src(nx, ny, b, j, i):
    if u_int(nx, ny, j, i): return (j, i)
    W, E, S, N = i == 0, i == nx - 2, j == 0, j == ny - 1
    if W and S: t = pick(b["uS"], b["uW"])
    elif E and S: t = pick(b["uS"], b["uE"])
    elif W and N: t = pick(b["uN"], b["uW"])
    elif E and N: t = pick(b["uN"], b["uE"])
    elif W: t = b["uW"]
    elif E: t = b["uE"]
    elif S: t = b["uS"]
    else: t = b["uN"]
    if t == ZERO: return None
    if t == INF: return ((1 if S else (ny - 2 if N else j)), (1 if W else (nx - 3 if E else i)))
    return ((ny - 2 if S else (1 if N else j)), (nx - 3 if W else (1 if E else i)))
def v_src(nx, ny, b, j, i):
    if v_int(nx, ny, j, i): return (j, i)
    W, E, S, N = i == 0, i == nx - 1, j == 0, j == ny - 2
    if W and S: t = pick(b["vS"], b["vW"])
    elif E and S: t = pick(b["vS"], b["vE"])
    elif W and N: t = pick(b["vN"], b["vW"])
    elif E and N: t = pick(b["vN"], b["vE"])
    elif W: t = b["vW"]
    elif E: t = b["vE"]
    elif S: t = b["vS"]
    else: t = b["vN"]
    if t == ZERO: return None
    if t == INF: return ((1 if S else (ny - 3 if N else j)), (1 if W else (nx - 2 if E else i)))
    return ((ny - 3 if S else (1 if N else j)), (nx - 2 if W else (1 if E else i)))
def ghosts_u(nx, ny, b, j, i):
    W, E, S, N = i == 1, i == nx - 3, j == 1, j == ny - 2
    out = set()
    if W and b["uW"] == INF: out.add((j, 0))
    if E and b["uE"] == INF: out.add((j, nx - 2))
    if S and b["uS"] == INF: out.add((0, i))
    if N and b["uN"] == INF: out.add((ny - 1, i))
    if W and S and pick(b["uS"], b["uW"]) == INF: out.add((0, 0))
    if E and S and pick(b["uS"], b["uE"]) == INF: out.add((0, nx - 2))
    if W and N and pick(b["uN"], b["uW"]) == INF: out.add((ny - 1, 0))
    if E and N and pick(b["uN"], b["uE"]) == INF: out.add((ny - 1, nx - 2))
    return out
def ghosts_v(nx, ny, b, j, i):
    W, E, S, N = i == 1, i == nx - 2, j == 1, j == ny - 3
    out = set()
    if W and b["vW"] == INF: out.add((j, 0))
    if E and b["vE"] == INF: out.add((j, nx - 1))
    if S and b["vS"] == INF: out.add((0, i))
    if N and b["vN"] == INF: out.add((ny - 2, i))
    if W and S and pick(b["vS"], b["vW"]) == INF: out.add((0, 0))
    if E and S and pick(b["vS"], b["vE"]) == INF: out.add((0, nx - 1))
    if W and N and pick(b["vN"], b["vW"]) == INF: out.add((ny - 2, 0))
    if E and N and pick(b["vN"], b["vE"]) == INF: out.add((ny - 2, nx - 1))
    return out

def test_direct_rule_writes_exactly_the_mapped_ghosts():
    keys = ["uW", "uE", "uS", "uN", "vW", "vE", "vS", "vN"]
    n = 0
    for combo in itertools.product([ZERO, INF], repeat=8):
        b = dict(zip(keys, combo))
        for nx, ny in ((5, 5), (6, 9), (9, 6), (12, 17)):
            # u: every boundary unknown in the u grid, grouped by source
            want = {}
            for j in range(ny):
                for i in range(nx - 1):
                    if not u_int(nx, ny, j, i):
                        s = u_src(nx, ny, b, j, i)
                        if s is not None:
                            assert u_int(nx, ny, *s), (b, nx, ny, j, i, s)
                            want.setdefault(s, set()).add((j, i))
            for j in range(ny):
                for i in range(nx - 1):
                    if u_int(nx, ny, j, i):
                        assert ghosts_u(nx, ny, b, j, i) == want.get((j, i), set()), ("u", b, nx, ny, j, i)
                        n += 1
            want = {}
            for j in range(ny - 1):
                for i in range(nx):
                    if not v_int(nx, ny, j, i):
                        s = v_src(nx, ny, b, j, i)
                        if s is not None:
                            assert v_int(nx, ny, *s)
                            want.setdefault(s, set()).add((j, i))
            for j in range(ny - 1):
                for i in range(nx):
                    if v_int(nx, ny, j, i):
                        assert ghosts_v(nx, ny, b, j, i) == want.get((j, i), set()), ("v", b, nx, ny, j, i)
                        n += 1
    assert n > 0


def test_outside_reads_map_back_to_the_row():
    keys = ["uW", "uE", "uS", "uN", "vW", "vE", "vS", "vN"]
    # the premise: a row's outside same-component neighbours map back to the row itself (or to zero)
    m = 0
    for combo in itertools.product([ZERO, INF], repeat=8):
        b = dict(zip(keys, combo))
        for nx, ny in ((5, 5), (6, 9), (9, 6), (12, 17)):
            for j in range(ny):
                for i in range(nx - 1):
                    if not u_int(nx, ny, j, i): continue
                    for (jj, ii) in ((j, i + 1), (j, i - 1), (j + 1, i), (j - 1, i)):
                        if not u_int(nx, ny, jj, ii):
                            s = u_src(nx, ny, b, jj, ii)
                            assert s is None or s == (j, i), ("u", b, nx, ny, (j, i), (jj, ii), s)
                            m += 1
            for j in range(ny - 1):
                for i in range(nx):
                    if not v_int(nx, ny, j, i): continue
                    for (jj, ii) in ((j + 1, i), (j - 1, i), (j, i + 1), (j, i - 1)):
                        if not v_int(nx, ny, jj, ii):
                            s = v_src(nx, ny, b, jj, ii)
                            assert s is None or s == (j, i), ("v", b, nx, ny, (j, i), (jj, ii), s)
                            m += 1
    assert m > 0
