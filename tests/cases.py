"""Seeded test instances shared by the CPU and GPU tests."""
from __future__ import annotations

from vfb_b200 import synth


def random_instance(seed: int, num_vars: int, n_pos: int, n_neg: int, lengths, max_size: int,
                    p: float = 0.5, rlx_type: int = 3) -> synth.Instance:
    """Unlabelled random traces (no planted formula); lengths: int or list per trace."""
    rng = synth.Rng(seed)
    n = n_pos + n_neg
    lens = lengths if isinstance(lengths, list) else [lengths] * n
    traces = []
    for i in range(n):
        traces.append((lens[i], [rng.bernoulli_word(lens[i], p) for _ in range(num_vars)]))
    return synth.Instance(num_vars, traces[:n_pos], traces[n_pos:], max_size,
                          [f"p{v}" for v in range(num_vars)], None, rlx_type, f"rand{seed}")


def small_exact_cases():
    """Instances with at most 126 trace bits (exact keys), minimal size <= ~7."""
    out = [synth.config_small()]
    for s in range(12):
        rng = synth.Rng(1000 + s)
        a = 1 + rng.below(3)
        npos = 1 + rng.below(3)
        nneg = 1 + rng.below(3)
        lens = [1 + rng.below(6) for _ in range(npos + nneg)]
        out.append(random_instance(2000 + s, a, npos, nneg, lens, 7))
    return out


def relaxed_cases(rlx_type: int):
    """Instances with more than 126 trace bits (relaxed keys)."""
    out = []
    for s in range(4):
        rng = synth.Rng(3000 + s)
        a = 2 + rng.below(2)
        npos = 4 + rng.below(4)
        nneg = 4 + rng.below(4)
        lens = [8 + rng.below(17) for _ in range(npos + nneg)]
        out.append(random_instance(4000 + s, a, npos, nneg, lens, 6, rlx_type=rlx_type))
    return out


def planted_cases(count: int = 6, max_size_extra: int = 2):
    """Planted-formula instances (labels from a uniformly drawn formula)."""
    out = []
    for s in range(count):
        rng = synth.Rng(5000 + s)
        a = 2 + rng.below(3)
        size = 4 + rng.below(4)
        t = 6 + rng.below(20)
        npos = t // 2
        inst = synth.planted_instance(rng, a, size, npos, t - npos, (4, 32), 0.5,
                                      size + max_size_extra, name=f"planted{s}")
        out.append(inst)
    return out


def unsatisfiable_cases(seeds=(4242, 4243, 4244, 4245)):
    """Instances with a positive trace equal to a negative one: nothing solves
    them, so every level up to max size 8 is built (about 200k rows each)."""
    out = []
    for seed in seeds:
        inst = random_instance(seed, 4, 5, 5, 16, 8)
        inst.neg[0] = inst.pos[0]
        out.append(inst)
    return out


def smallest_solo_budget(probs, want, sizes_mb=(32, 48, 64, 96, 128, 192, 256)):
    """The smallest device budget (bytes) under which every problem, solved
    alone in a fresh context, returns the result in want (GPU only)."""
    import vfb_b200
    key = lambda r: (r.status, r.size, r.rpn, r.level_rows, r.level_cands)  # noqa: E731
    for mb in sizes_mb:
        with vfb_b200.Engine(mem_limit_bytes=mb << 20) as eng:
            if all(key(eng.solve(p)) == key(w) for p, w in zip(probs, want)):
                return mb << 20
    return None


def mirrored_cases(count: int = 8, num_vars: int = 5, length: int = 18, max_size: int = 6):
    """Instances whose relaxed (hash) keys collide for every formula and its
    mirror (propositions 0 and 1 swapped): traces come in pairs, the second
    the first with propositions 0 and 1 exchanged, both in the same half of the
    traces (hash keys fold each half with XOR, so the pair's words cancel
    into the same key).  Traces 0, 1 are positive and their mirrors 2, 3
    negative, so a formula and its mirror never both solve: whenever the
    first solving formula's mirror comes earlier in the order, the first
    solving candidate does not own its key."""
    out = []
    for s in range(count):
        rng = synth.Rng(7000 + s)
        base = [[rng.bernoulli_word(length, 0.5) for _ in range(num_vars)] for _ in range(4)]
        def mirror(w):
            m = list(w)
            m[0], m[1] = w[1], w[0]
            return m
        # halves of 8 traces: {0, 1, 2, 3} and {4, 5, 6, 7}
        traces = [base[0], base[1], mirror(base[0]), mirror(base[1]),
                  base[2], mirror(base[2]), base[3], mirror(base[3])]
        tr = [(length, w) for w in traces]
        out.append(synth.Instance(num_vars, tr[:2], tr[2:], max_size,
                                  [f"p{v}" for v in range(num_vars)], None, 3, f"mirror{s}"))
    return out
