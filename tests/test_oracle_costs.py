"""The oracle's weighted order (operator costs c1..c8 and NegType of LTL_BS)
against an independent restatement: the minimal cost of a solution, found by
plain enumeration of characteristic sets level by level."""
from tests import cases
import oracle

OPS = "~&|XFGU"


def _brute_min_cost(inst, costs, neg_type, kmax):
    T, lens, words, npos = inst.num_traces, inst.lengths(), inst.atom_words(), len(inst.pos)

    def mask(L):
        return (1 << L) - 1

    def sfx(w):
        for s in (1, 2, 4, 8, 16, 32):
            w |= w >> s
        return w

    def app(op, lw, rw):
        out = []
        for t in range(T):
            L, a, b = lens[t], lw[t], rw[t] if rw else 0
            if op == "~":
                v = ~a & mask(L)
            elif op == "&":
                v = a & b
            elif op == "|":
                v = a | b
            elif op == "X":
                v = a >> 1
            elif op == "F":
                v = sfx(a)
            elif op == "G":
                v = a & ~sfx(~a & mask(L))
            else:   # U by its recurrence, from the last step backwards
                v = 0
                for i in range(L - 1, -1, -1):
                    v |= (((b >> i) & 1) or (((a >> i) & 1) and ((v >> (i + 1)) & 1))) << i
            out.append(v)
        return tuple(out)

    def sol(cs):
        return all((cs[t] & 1) == (1 if t < npos else 0) for t in range(T))

    c1, w = costs[0], dict(zip(OPS, costs[1:]))
    levels, seen = {c1: []}, set()
    for v in range(inst.num_vars):
        cs = tuple(words[v])
        if sol(cs):
            return c1
        seen.add(cs)
        levels[c1].append(cs)
    for k in range(c1 + 1, kmax + 1):
        levels[k] = []
        for op in OPS:
            pairs = []
            if op in "~XFG":
                L = k - w[op]
                if L < c1 or (op == "~" and neg_type == 2 and L != c1):
                    continue
                pairs = [(a, None) for a in levels.get(L, [])]
            else:
                i = c1
                while True:
                    j = k - w[op] - i
                    if j < c1 or (op != "U" and i > j):
                        break
                    pairs += [(a, b) for a in levels.get(i, []) for b in levels.get(j, [])]
                    i += 1
            for a, b in pairs:
                cs = app(op, a, b)
                if cs in seen:
                    continue
                seen.add(cs)
                levels[k].append(cs)
                if sol(cs):
                    return k
    return None


def test_weighted_order_finds_minimal_cost():
    found = 0
    for seed in range(9000, 9020):
        inst = cases.random_instance(seed, 2, 3, 3, [3, 4, 5, 3, 4, 5], 9)
        for costs, neg in [([1, 2, 2, 2, 1, 1, 1, 3], 1), ([2, 1, 3, 3, 2, 2, 2, 2], 2)]:
            r = oracle.solve(oracle.Problem.from_instance(inst, costs=costs, neg_type=neg))
            want = _brute_min_cost(inst, costs, neg, 9)
            if r["status"] == oracle.FOUND:
                ok, _ = oracle.eval_rpn(oracle.Problem.from_instance(inst), r["rpn"])
                cost = sum(costs[0] if isinstance(t, int) else costs[1 + OPS.index(t)] for t in r["rpn"])
                assert ok == 1 and cost == r["size"] == want
                found += 1
            else:
                assert want is None
    assert found >= 20


def test_unit_costs_are_the_size_order():
    for inst in cases.small_exact_cases()[:6]:
        a = oracle.solve(oracle.Problem.from_instance(inst))
        b = oracle.solve(oracle.Problem.from_instance(inst, costs=[1] * 8, neg_type=1))
        assert (a["status"], a["size"], a["rpn"], a["level_rows"]) == (b["status"], b["size"], b["rpn"], b["level_rows"])
