"""A host model of assign_resident_kernel's control flow (onedal_b200/csrc/kmb_assign_plain.cu),
checked on the CPU before any GPU runs it.

The kernel's two warp groups take turns at the FMA pipe through named barriers 1 and
2, meet at CTA barriers around each chunk's centroid load, at a group barrier after a
tile's last contraction (one-stage form), and consume TMA row loads in the order their
single issuing thread issued them. The model replays each group's sequence of those
operations for one CTA -- the same loop bounds, tile indices, next-tile rule, stage and
parity bookkeeping as the kernel -- and schedules the two groups against each other.
It checks, for row counts around the tile and step sizes, grids that wrap, one or
several chunks, one or two stages and several block sizes:

* no deadlock: every turn wait is matched by the other group's hand-over, with never
  more than one hand-over pending on a barrier (a second arrival would complete the
  barrier without the waiting group), and both groups reach every CTA barrier;
* every load a group issues is waited for, in order, at the stage and phase parity the
  consumer computes, and every tile is the one it contracts;
* over the grid, every 64-row tile is contracted exactly once per 256-cluster pass.
"""
import pytest

R = 64  # rows per tile


def group_program(g, n, grid, b, kres, kchunk, bt, stages):
    n_tiles = (n + R - 1) // R
    par_tiles = (n_tiles - g + 1) // 2
    par_tiles0 = (n_tiles + 1) // 2
    my_tiles = (par_tiles - b + grid - 1) // grid if par_tiles > b else 0
    steps = (par_tiles0 - b + grid - 1) // grid if par_tiles0 > b else 0
    n_chunks = (kres + kchunk - 1) // kchunk
    total_turns = steps * (kres // 256)
    ops, m_issue, m_wait, turn = [], 0, 0, 0
    if my_tiles > 0:
        ops.append(("issue", 0, 0))
        m_issue = 1
    for blk in range((steps + bt - 1) // bt):
        u_n = min(bt, steps - blk * bt)
        for q in range(n_chunks):
            if n_chunks > 1 and (blk > 0 or q > 0):
                ops += [("cta",), ("cta",)]
            ppc = min(kchunk, kres - q * kchunk) // 256
            for ut in range(u_n):
                lt = blk * bt + ut
                has = lt < my_tiles
                if ut + 1 < u_n and lt + 1 < my_tiles:
                    nxt = lt + 1
                elif q + 1 < n_chunks:
                    nxt = blk * bt
                else:
                    nxt = (blk + 1) * bt
                nxt_has = has and nxt < my_tiles
                stage, parity = m_wait % stages, (m_wait // stages) & 1
                if has:
                    m_wait += 1
                for p in range(ppc):
                    if g == 0:
                        if turn > 0:
                            ops.append(("wait", 1))
                    else:
                        ops.append(("wait", 2))
                    if p == 0 and has:
                        if stages == 2 and nxt_has:
                            ops.append(("issue", m_issue % 2, nxt))
                            m_issue += 1
                        ops.append(("consume", stage, parity, lt))
                    last = p + 1 == ppc
                    if g == 0:
                        ops.append(("give", 2))
                    elif turn + 1 < total_turns:
                        ops.append(("give", 1))
                    if stages == 1 and last and nxt_has:
                        ops.append(("issue", 0, nxt))
                        m_issue += 1
                    if has:
                        ops.append(("use", lt, q, p))
                    turn += 1
    ops.append(("cta",))
    return ops


def run_cta(n, grid, b, kres, kchunk, bt, stages):
    progs = [group_program(g, n, grid, b, kres, kchunk, bt, stages) for g in range(2)]
    pc = [0, 0]
    gives, waits = {1: 0, 2: 0}, {1: 0, 2: 0}
    arrived, blocked = [0, 0], [False, False]
    loads = [[[], []], [[], []]]
    consumed = [[0, 0], [0, 0]]
    used = [[], []]
    while pc[0] < len(progs[0]) or pc[1] < len(progs[1]):
        progressed = False
        for g in range(2):
            while pc[g] < len(progs[g]):
                op = progs[g][pc[g]]
                if op[0] == "wait":
                    if gives[op[1]] <= waits[op[1]]:
                        break
                    waits[op[1]] += 1
                elif op[0] == "give":
                    gives[op[1]] += 1
                    assert gives[op[1]] <= waits[op[1]] + 1, "two hand-overs pending on one barrier"
                elif op[0] == "cta":
                    if not blocked[g]:
                        arrived[g] += 1
                        blocked[g] = True
                        progressed = True
                    if arrived[1 - g] < arrived[g]:
                        break
                    blocked[g] = False
                elif op[0] == "issue":
                    loads[g][op[1]].append(op[2])
                elif op[0] == "consume":
                    st, par, lt = op[1:]
                    k = consumed[g][st]
                    assert k < len(loads[g][st]), "waited for a load never issued"
                    assert loads[g][st][k] == lt and (k & 1) == par, "wrong tile or parity"
                    consumed[g][st] += 1
                elif op[0] == "use":
                    used[g].append(op[1:])
                pc[g] += 1
                progressed = True
        assert progressed, f"deadlock at {pc}"
    assert gives == waits
    for g in range(2):
        for st in range(2):
            assert consumed[g][st] == len(loads[g][st]), "a load left in flight"
    return used


@pytest.mark.parametrize("kres,kchunk,bts", [(256, 256, [1]), (768, 768, [1]), (1024, 256, [8, 4]),
                                             (1024, 512, [8, 3]), (1280, 512, [4])])
@pytest.mark.parametrize("stages", [1, 2])
@pytest.mark.parametrize("n", [1, 63, 64, 65, 128, 129, 4097, 148 * 128 * 3 + 65])
def test_resident_control_flow(n, stages, kres, kchunk, bts):
    n_tiles = (n + R - 1) // R
    for grid_max in (148, 3):
        grid = min((n + 127) // 128, grid_max)
        for bt in bts:
            seen = {}
            for b in range(grid):
                used = run_cta(n, grid, b, kres, kchunk, bt, stages)
                for g in range(2):
                    for lt, q, p in used[g]:
                        seen.setdefault(2 * (b + lt * grid) + g, []).append((q, p))
            assert sorted(seen) == list(range(n_tiles))
            assert all(len(v) == kres // 256 and len(set(v)) == len(v) for v in seen.values())
