"""Standalone runs of the hot-path workloads at their benchmark sizes, for
profilers and quick timing: each case builds its seeded inputs on cuda:0,
runs the operation `--reps` times through the public Python API and prints
the median CUDA-event time.

    python -m lattica_b200.cases round --reps 24     # LaBRADOR prover round
    python -m lattica_b200.cases gram --reps 4       # r x r Gram, r = 64, n = 2048
    python -m lattica_b200.cases commit --reps 4     # 16 x 2048 matrix times 64 witnesses
    python -m lattica_b200.cases garbage_h --reps 4  # h = sym(Phi S^T) / 2, r = 64, n = 2048
    python -m lattica_b200.cases amortize --reps 4   # z = sum_i c_i s_i, r = 64, n = 2048
    python -m lattica_b200.cases jl_evals --reps 4   # 256 conjugated JL evaluations, same witness
    python -m lattica_b200.cases ntt256 --reps 4     # d = 256 products, 2^20 polys at q'
    python -m lattica_b200.cases commit_plain --reps 5  # A 8 x 64 from a seed, 64 ternary witnesses
    python -m lattica_b200.cases jl_extract --reps 3 --parts 16  # JL p + int8 entries
    python -m lattica_b200.cases batch --parts 4096 --engine point_major  # uneven batched commits
                                                    # (engines: point_major, tensor, cuda_core)
    python -m lattica_b200.cases gram_batch --parts 16  # Gram of 16 witnesses, r in 8..64, n = 1024
    python -m lattica_b200.cases ring_round --reps 5    # the round at q = 2^32 - 5 (no NTT)

Sizes: r = 64 witness vectors of n = 2048 polys (d = 64, coefficients in
[-2^11, 2^11], as Montgomery words), kappa = 16, JL 256 rows, base 2^8 x 4
limbs; q = 4294966657 (q' = 4294962689 for d = 256)."""
import argparse
import statistics

Q = 4294966657
Q256 = 4294962689


def _witness(torch, dev, g, q, shape):
    coeffs = torch.randint(-2048, 2049, shape, dtype=torch.int64, device=dev, generator=g) % q
    return ((coeffs * ((1 << 32) % q)) % q).to(torch.int32)


def _uniform(torch, dev, g, q, shape):
    return torch.randint(0, q, shape, dtype=torch.int64, device=dev, generator=g).to(torch.int32)


def _commit_plain(torch, dev, g, plan):
    """The plain Ajtai commitment: A 8 x 64 expanded from a seed, 64 witnesses of
    64 ternary polynomials, through grid_gpu_commit_dev."""
    from lattica_b200 import _lib
    from lattica_b200.commit import PreparedMatrix
    from lattica_b200.labrador import sample_uniform_polys
    rows, cols, batch = 8, 64, 64
    lib = _lib.load()
    A = sample_uniform_polys(plan, bytes(range(100, 132)), rows * cols).reshape(rows, cols, 64)
    M = PreparedMatrix(plan, A, rows, cols)
    tern = torch.randint(-1, 2, (batch * cols, 64), dtype=torch.int64, device=dev, generator=g)
    s = ((tern % Q) * ((1 << 32) % Q) % Q).to(torch.int32)
    t = torch.empty((batch * rows, 64), dtype=torch.int32, device=dev)
    ws = torch.empty(max(256, M.workspace_bytes(batch)), dtype=torch.uint8, device=dev)

    def run():
        st = torch.cuda.current_stream(dev).cuda_stream
        code = lib.grid_gpu_commit_dev(M.handle, s.data_ptr(), batch, t.data_ptr(), ws.data_ptr(),
                                       ws.numel(), st)
        if code:
            raise RuntimeError(f"grid_gpu_commit_dev: {code}")
    run.keep = (M, A)
    return run


def _jl_extract(torch, dev, g, plan, parts, n):
    """JL projection of `parts` witness vectors (n polys, d = 64) by 256 rows,
    with the int8 entries, through grid_gpu_jl_project_dev."""
    import ctypes as C
    from lattica_b200 import _lib
    lib = _lib.load()
    S = _uniform(torch, dev, g, Q, (parts, n * 64))
    seed = (C.c_uint8 * 32)(*range(32))
    nb = C.c_size_t()
    lib.grid_gpu_jl_workspace(256, C.byref(nb))
    ws = torch.empty(max(256, nb.value), dtype=torch.uint8, device=dev)
    p = torch.empty(256, dtype=torch.int32, device=dev)
    flat = torch.empty(256 * parts * n * 64, dtype=torch.int8, device=dev)

    def run():
        st = torch.cuda.current_stream(dev).cuda_stream
        code = lib.grid_gpu_jl_project_dev(plan.handle, seed, 256, S.data_ptr(), parts, n * 64, 64,
                                           p.data_ptr(), flat.data_ptr(), ws.data_ptr(),
                                           ws.numel(), st)
        if code:
            raise RuntimeError(f"grid_gpu_jl_project_dev: {code}")
    return run


def _batch(torch, dev, g, plan, num, engine):
    """Uneven batched commits: num instances, n log-uniform in [64, 8192], rank
    in {8, 16, 32}, one m x 8192 matrix per rank; engine: tensor, cuda_core or
    point_major."""
    from lattica_b200 import _lib
    from lattica_b200.batch import UnevenCommitBatch, sample_uneven_instances
    from lattica_b200.commit import PreparedMatrix
    mats = [PreparedMatrix(plan, _uniform(torch, dev, g, Q, (m, 8192, 64)), m, 8192)
            for m in (8, 16, 32)]
    items, s_polys, t_polys = sample_uneven_instances(num, 7)
    tern = torch.randint(-1, 2, (s_polys, 64), dtype=torch.int64, device=dev, generator=g)
    s = ((tern % Q) * ((1 << 32) % Q) % Q).to(torch.int32)
    t = torch.empty((t_polys, 64), dtype=torch.int32, device=dev)
    batch = UnevenCommitBatch(plan, mats, items)
    engines = {"tensor": _lib.ENGINE_TENSOR, "cuda_core": _lib.ENGINE_CUDA_CORE,
               "point_major": _lib.ENGINE_POINT_MAJOR}
    batch.set_config(4096, 0, engines[engine])
    run = lambda: batch.commit_dev(s, t)
    run.keep = (mats, batch)
    return run


def _gram_batch(torch, dev, g, plan, count):
    """Gram matrices of `count` witnesses, r cycling over 8, 16, 32, 64, n = 1024,
    through grid_gpu_batch_gram_dev."""
    from lattica_b200.labrador import compute_garbage_g_batch
    items, off = [], 0
    for i in range(count):
        r = (8, 16, 32, 64)[i % 4]
        items.append((off, r, 1024))
        off += r * 1024
    pool = _witness(torch, dev, g, Q, (off, 64))
    return lambda: compute_garbage_g_batch(plan, pool, items)


def build(case: str, parts: int = 64, engine: str = "tensor"):
    """Returns a zero-argument callable that runs one instance of `case`
    (`parts`: witness vectors of jl_extract, instances of batch and gram_batch)."""
    import torch
    from lattica_b200 import TwistedNttPlan
    from lattica_b200.labrador import (CommitKey, JLMatrix, amortize_witness, compute_garbage_g,
                                       compute_garbage_h, prover_round_dev)
    dev = torch.device("cuda:0")
    g = torch.Generator(device=dev).manual_seed(5)
    r, n, kappa = 64, 2048, 16
    if case == "ntt256":
        plan = TwistedNttPlan(Q256, 256)
        a = _uniform(torch, dev, g, Q256, (1 << 20, 256))
        b = _uniform(torch, dev, g, Q256, (1 << 20, 256))
        return lambda: plan.ntt_mul_inverse(a, b)
    if case == "ring_round":
        from lattica_b200.ntt import RingPlan
        q = 4294967291  # 2^32 - 5: three auxiliary NTT primes, exact reconstruction
        plan = RingPlan(q, 64)
        wit = _witness(torch, dev, g, q, (r, n, 64))
        key = CommitKey(plan, _uniform(torch, dev, g, q, (kappa, n, 64)), kappa, n)
        seed = bytes(range(32))
        return lambda: prover_round_dev(key, wit, 256, 4, 256, 4, seed, 256)
    plan = TwistedNttPlan(Q, 64)
    if case == "commit_plain":
        return _commit_plain(torch, dev, g, plan)
    if case == "jl_extract":
        return _jl_extract(torch, dev, g, plan, parts, n)
    if case == "batch":
        return _batch(torch, dev, g, plan, parts, engine)
    if case == "gram_batch":
        return _gram_batch(torch, dev, g, plan, parts)
    wit = _witness(torch, dev, g, Q, (r, n, 64))
    if case == "gram":
        return lambda: compute_garbage_g(plan, wit)
    if case == "garbage_h":
        phis = _uniform(torch, dev, g, Q, (r, n, 64))
        return lambda: compute_garbage_h(plan, wit, phis)
    if case == "jl_evals":
        jl = JLMatrix(bytes(range(32)), 256, n * 64)
        flat = wit.reshape(r, n * 64)
        return lambda: jl.conjugated_evals(plan, flat, r, 64)
    if case == "amortize":
        chal = _uniform(torch, dev, g, Q, (r, 64))
        return lambda: amortize_witness(plan, wit, chal)
    key = CommitKey(plan, _uniform(torch, dev, g, Q, (kappa, n, 64)), kappa, n)
    if case == "commit":
        return lambda: key.inner_commit_slice(wit)
    if case == "round":
        seed = bytes(range(32))
        return lambda: prover_round_dev(key, wit, 256, 4, 256, 4, seed, 256)
    raise ValueError(f"unknown case {case!r}")


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("case", choices=["round", "gram", "garbage_h", "amortize", "jl_evals", "commit",
                                       "ntt256", "commit_plain", "jl_extract", "batch",
                                       "gram_batch", "ring_round"])
    ap.add_argument("--reps", type=int, default=4)
    ap.add_argument("--parts", type=int, default=64,
                    help="witness vectors (jl_extract), instances (batch, gram_batch)")
    ap.add_argument("--engine", choices=["tensor", "cuda_core", "point_major"], default="tensor",
                    help="grouped-product engine of the batch case")
    args = ap.parse_args(argv)
    import torch
    fn = build(args.case, args.parts, args.engine)
    fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    print(f"{args.case}: {len(times)} runs, median {statistics.median(times):.4f} ms")


if __name__ == "__main__":
    main()
