"""CPU models of kernel index mappings:

* the element placement of the T-threads-per-polynomial transform stages
  (`fwdT_stages` / `invT_stages` in lattica_b200/csrc/ntt.cu) at d = 64,
  T = 8, as the one-launch commitment uses them, against the
  one-thread-per-polynomial stages (`fwd1_stages` / `inv1_stages`);
* the 4 x 4 byte transpose across a lane quad in the JL projection kernel
  that writes the int8 entries (`jl_tc_kernel<true, true>` in jl.cu);
* the instance-row copies of the grouped point-major product
  (`batch_pm_kernel` in grouped_pm.cu): which rows each chunk copies or
  zero-fills, over rotating shared-memory slots;
* the mbarrier protocols of the tensor-core transform (`ntt_tc_kernel`) and of
  the grouped point-major product: parity waits never meet a barrier two
  phases past the awaited one, and no buffer, slot or accumulator is reused
  early, over random interleavings of the roles and of copy / MMA completions.

The models restate the kernels' index arithmetic with exact arithmetic mod q
and arbitrary twiddle values, so they check data movement, not the field."""
import random

Q = 4294966657


def _brv(x, bits):
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


def _log2(x):
    return x.bit_length() - 1


def _one_thread_forward(inp, fw, d):
    x = list(inp)
    ln = d // 2
    while ln >= 1:
        for g in range(d // (2 * ln)):
            k = d // (2 * ln) + g
            for j in range(g * 2 * ln, g * 2 * ln + ln):
                u, v = x[j], x[j + ln]
                t = fw[k] * v % Q
                x[j], x[j + ln] = (u + t) % Q, (u - t) % Q
        ln //= 2
    return {s: x[_brv(s, _log2(d))] for s in range(d)}  # slot -> value


def _threads_forward(inp, fw, d, T):
    E, logd = d // T, _log2(d)
    X = [[inp[4 * (T * m + t) + s] for m in range(E // 4) for s in range(4)] for t in range(T)]
    ln = d // 2
    while ln >= 1:
        l2 = _log2(2 * ln)
        if ln >= 4 * T:
            step = ln // T
            for t in range(T):
                for e in range(E):
                    if e & step == 0:
                        k = d // (2 * ln) + ((4 * T * (e >> 2)) >> l2)
                        u, v = X[t][e], X[t][e + step]
                        w = fw[k] * v % Q
                        X[t][e], X[t][e + step] = (u + w) % Q, (u - w) % Q
        elif ln >= 4:
            M = ln // 4

            def mine(t, e):
                k = d // (2 * ln) + ((4 * T * (e >> 2) + 4 * t) >> l2)
                return fw[k] * X[t][e] % Q if t & M else X[t][e]
            X = [[(mine(t ^ M, e) - mine(t, e)) % Q if t & M else (mine(t, e) + mine(t ^ M, e)) % Q
                  for e in range(E)] for t in range(T)]
        else:
            for t in range(T):
                for e in range(E):
                    if e & ln == 0:
                        k = d // (2 * ln) + ((4 * T * (e >> 2) + 4 * t + (e & 3)) >> l2)
                        u, v = X[t][e], X[t][e + ln]
                        w = fw[k] * v % Q
                        X[t][e], X[t][e + ln] = (u + w) % Q, (u - w) % Q
        ln //= 2
    out = {}
    for t in range(T):
        for e in range(E):
            i = 4 * T * (e >> 2) + (e & 3)
            out[_brv(i, logd) | _brv(4 * t, logd)] = X[t][e]
    return out


def _one_thread_inverse(slots, iw, ninv, iw1n, d):
    x = [0] * d
    for s in range(d):
        x[_brv(s, _log2(d))] = slots[s]
    ln = 1
    while ln <= d // 2:
        if ln == d // 2:
            for j in range(ln):
                u, v = x[j], x[j + ln]
                x[j], x[j + ln] = (u + v) * ninv % Q, (u - v) * iw1n % Q
        else:
            for g in range(d // (2 * ln)):
                k = d // (2 * ln) + g
                for j in range(g * 2 * ln, g * 2 * ln + ln):
                    u, v = x[j], x[j + ln]
                    x[j], x[j + ln] = (u + v) % Q, (u - v) * iw[k] % Q
        ln *= 2
    return x


def _threads_inverse(slots, iw, ninv, iw1n, d, T):
    E, logd = d // T, _log2(d)
    X = [[slots[_brv(4 * T * (e >> 2) + (e & 3), logd) | _brv(4 * t, logd)] for e in range(E)]
         for t in range(T)]
    ln = 1
    while ln <= d // 2:
        l2 = _log2(2 * ln)
        if ln == d // 2:
            step = ln // T
            for t in range(T):
                for e in range(E):
                    if e & step == 0:
                        u, v = X[t][e], X[t][e + step]
                        X[t][e], X[t][e + step] = (u + v) * ninv % Q, (u - v) * iw1n % Q
        elif ln >= 4 * T:
            step = ln // T
            for t in range(T):
                for e in range(E):
                    if e & step == 0:
                        k = d // (2 * ln) + ((4 * T * (e >> 2)) >> l2)
                        u, v = X[t][e], X[t][e + step]
                        X[t][e], X[t][e + step] = (u + v) % Q, (u - v) * iw[k] % Q
        elif ln >= 4:
            M = ln // 4
            new = [row[:] for row in X]
            for t in range(T):
                for e in range(E):
                    k = d // (2 * ln) + ((4 * T * (e >> 2) + 4 * t) >> l2)
                    other = X[t ^ M][e]
                    s = (other - X[t][e]) % Q if t & M else (X[t][e] + other) % Q
                    new[t][e] = s * iw[k] % Q if t & M else s
            X = new
        else:
            for t in range(T):
                for e in range(E):
                    if e & ln == 0:
                        k = d // (2 * ln) + ((4 * T * (e >> 2) + 4 * t + (e & 3)) >> l2)
                        u, v = X[t][e], X[t][e + ln]
                        X[t][e], X[t][e + ln] = (u + v) % Q, (u - v) * iw[k] % Q
        ln *= 2
    out = [0] * d
    for t in range(T):
        for m in range(E // 4):
            for s in range(4):
                out[4 * (T * m + t) + s] = X[t][4 * m + s]
    return out


def test_eight_thread_transform_places_every_value_like_one_thread():
    rng = random.Random(3)
    for d, T in ((64, 8), (64, 4), (128, 2), (256, 4)):
        for _ in range(4):
            fw = [rng.randrange(Q) for _ in range(d)]
            iw = [rng.randrange(Q) for _ in range(d)]
            ninv, iw1n = rng.randrange(Q), rng.randrange(Q)
            inp = [rng.randrange(Q) for _ in range(d)]
            assert _threads_forward(inp, fw, d, T) == _one_thread_forward(inp, fw, d), (d, T)
            slots = [rng.randrange(Q) for _ in range(d)]
            assert (_threads_inverse(slots, iw, ninv, iw1n, d, T) ==
                    _one_thread_inverse(slots, iw, ninv, iw1n, d)), (d, T)


def _byte_perm(x, y, s):
    b = [(x >> (8 * i)) & 0xFF for i in range(4)] + [(y >> (8 * i)) & 0xFF for i in range(4)]
    return sum(b[(s >> (4 * i)) & 7] << (8 * i) for i in range(4))


def test_lane_quad_byte_transpose_of_jl_entries():
    """Lane u of a quad holds rows 4b..4b+3 of polynomial u as M' = M + 1 bytes;
    after the two exchanges lane r holds row 4b + r of polynomials 0..3 as int8 M."""
    rng = random.Random(5)
    for _ in range(500):
        M = [[rng.randint(0, 2) for _ in range(4)] for _ in range(4)]  # [poly u][row r] = M'
        words = [sum(M[u][r] << (8 * r) for r in range(4)) for u in range(4)]
        m = [((w + 0x7F7F7F7F) & 0xFFFFFFFF) ^ 0x80808080 for w in words]
        a = [_byte_perm(m[u], m[u ^ 1], 0x3715 if u & 1 else 0x6240) for u in range(4)]
        o = [_byte_perm(a[u], a[u ^ 2], 0x3276 if u & 2 else 0x5410) for u in range(4)]
        for r in range(4):
            for u in range(4):
                assert (o[r] >> (8 * u)) & 0xFF == (M[u][r] - 1) & 0xFF


def _sw128(row, c16):
    """Byte offset of 16-byte chunk c16 of `row` in a 128-byte-swizzled tile."""
    return (row >> 3) * 1024 + (row & 7) * 128 + ((c16 ^ (row & 7)) << 4)


def test_grouped_point_major_loader_keeps_live_rows_and_zeroes_finished_ones():
    """The copy bookkeeping of batch_pm_kernel (grouped_pm.cu): four loader
    warps of 32 instance rows, eight lanes per row and four rows per step; per
    chunk, rows still inside their length (a prefix: tiles are sorted longest
    first) are copied, rows that ran out since the slot last held this item are
    zero-filled, and the rest are left as they are. Slots rotate over chunks and
    items. Every stored row of every chunk must read its words inside the
    instance's padded columns, and hold exactly its words there, zero past n."""
    rng = random.Random(11)
    NSA, KCH = 4, 32
    slots = [[rng.randrange(1 << 32) for _ in range(128 * 32)] for _ in range(NSA)]  # old data
    gc = 0
    for item in range(40):
        count = rng.randint(1, 128)
        ns = sorted((rng.randint(1, 900) for _ in range(count)), reverse=True)
        kmax = ns[0]
        k_split = rng.choice([32, 64, 256, 1024])
        k0 = rng.randrange(0, kmax, 32) if kmax > 32 else 0
        k0 -= k0 % k_split
        k1 = min(kmax, k0 + k_split)
        padded = [(n + 127) // 128 * 128 for n in ns]
        value = lambda j, k: (j * 100003 + k * 7 + item) % (1 << 32)
        zeroed = [[32] * NSA for _ in range(4)]  # per loader warp, per slot
        for c in range((k1 - k0 + KCH - 1) // KCH):
            sl = gc % NSA
            kc = k0 + c * KCH
            tile = slots[sl]
            for lw in range(4):
                row0 = 32 * lw
                cw = max(0, min(count - row0, 32))
                J = sum(1 for jr in range(cw) if ns[row0 + jr] > kc)
                assert all(ns[row0 + jr] > kc for jr in range(J))  # a prefix
                zend = min(max(zeroed[lw][sl], J), cw)
                for s8 in range(8):
                    for lane in range(32):
                        r, q4 = lane >> 3, lane & 7
                        jr = 4 * s8 + r
                        if jr >= zend:
                            continue
                        j = row0 + jr
                        off = _sw128(j, q4) // 4
                        for w in range(4):
                            k = kc + 4 * q4 + w
                            if jr < J:  # 16 bytes of the instance's columns
                                assert k < padded[j]
                                tile[off + w] = value(j, k) if k < ns[j] else 0
                            else:
                                tile[off + w] = 0
                zeroed[lw][sl] = min(J, cw)
            for j in range(count):
                for kk in range(KCH):
                    k = kc + kk
                    word = tile[_sw128(j, kk >> 2) // 4 + (kk & 3)]
                    assert word == (value(j, k) if k < ns[j] else 0), (item, c, j, kk)
            gc += 1


def _transform_roles(n, two, old_loader_wait):
    """The waits and arrivals of ntt_tc_kernel's loader, MMA and epilogue
    roles for n tiles (two: the NTT -> product -> INTT mode). Each role is a
    generator of ('wait', barrier, phase index), ('arrive', barrier) and
    ('async', barrier) (a copy or MMA completion that lands later)."""
    lag = 3 if two else 2

    def loader():
        staged_seen = [0, 0]
        for t in range(n + lag):
            if old_loader_wait:
                if t >= 2 and t - 2 < n:
                    yield ("wait", "FDONE", t - 2)
            elif two and t == 1 and n > 0:
                yield ("wait", "FDONE", 0)
            if t >= lag:
                buf = t & 1
                yield ("wait", f"STAGED{buf}", staged_seen[buf])
                staged_seen[buf] += 1
            if t < n:
                if t >= 2:  # buffer t & 1 held tile t - 2: its forward must be done
                    yield ("check", "FDONE", t - 1)
                yield ("async", f"AFULL{t & 1}")

    def mma():
        def inverse(j):
            yield ("wait", "PREADY", j)
            if j >= 1:
                yield ("wait", "EREAD", j - 1)
            yield ("async", "IDONE")
        for j in range(n):
            yield ("wait", f"AFULL{j & 1}", j >> 1)
            if j >= 1:
                yield ("wait", "FREAD", j - 1)
            yield ("async", "FDONE")
            if two and j >= 1:
                yield from inverse(j - 1)
        if two and n > 0:
            yield from inverse(n - 1)

    def epilogue():
        def inverse_out(j):
            yield ("wait", "IDONE", j)
            yield ("arrive", "EREAD")
            yield ("arrive", f"STAGED{(j + 1) & 1}")
        for j in range(n):
            yield ("wait", "FDONE", j)
            yield ("arrive", "FREAD")
            if two:
                if j >= 1:
                    yield ("wait", "IDONE", j - 1)
                yield ("arrive", "PREADY")
                if j >= 1:
                    yield from inverse_out(j - 1)
            else:
                yield ("arrive", f"STAGED{j & 1}")
        if two and n > 0:
            yield from inverse_out(n - 1)

    return [loader(), mma(), epilogue()]


def _run_transform_model(n, two, old_loader_wait, rng):
    """Random interleaving with mbarrier parity semantics; returns the first
    wait that met its barrier two or more phases past the awaited one (where a
    parity test reads a completed phase as pending), or the first load into a
    buffer whose previous tile's forward transform had not completed, or None."""
    done = {}
    roles = _transform_roles(n, two, old_loader_wait)
    current = [next(r, None) for r in roles]
    pending = []  # async completions not landed yet
    while any(c is not None for c in current) or pending:
        choices = [("role", i) for i, c in enumerate(current) if c is not None]
        choices += [("land", i) for i in range(len(pending))]
        kind, i = rng.choice(choices)
        if kind == "land":
            bar = pending.pop(i)
            done[bar] = done.get(bar, 0) + 1
            continue
        op = current[i]
        if op[0] == "wait":
            completed = done.get(op[1], 0)
            if completed >= op[2] + 2:
                return op
            if completed <= op[2]:
                # blocked; if nothing else can move the model is stuck
                if not pending and all(c is None or c[0] == "wait" and done.get(c[1], 0) <= c[2]
                                       for c in current):
                    raise AssertionError(f"stuck at {current}")
                continue
        elif op[0] == "check":
            if done.get(op[1], 0) < op[2]:
                return op
        elif op[0] == "arrive":
            done[op[1]] = done.get(op[1], 0) + 1
        else:
            pending.append(op[1])
        current[i] = next(roles[i], None)
    return None


def test_transform_barrier_waits_never_alias_a_phase():
    """ntt_tc_kernel's waits are parity waits: each is correct only while its
    barrier is at most one phase past the awaited one. Over random
    interleavings of the three roles and of copy and MMA completions, no wait
    of the kernel as written ever meets an older phase, and no load refills a
    buffer before the forward transform of its previous tile. The loader's earlier
    wait for fwd(t - 2) did: with load t - 1 issued, fwd(t - 1) could complete
    before it polled."""
    rng = random.Random(5)
    for two in (False, True):
        for n in (1, 2, 3, 7):
            for _ in range(300):
                assert _run_transform_model(n, two, False, rng) is None, (two, n)
    hits = sum(_run_transform_model(7, False, True, rng) is not None for _ in range(300))
    assert hits > 0  # the model does find the old race


def _grouped_pm_roles(items, nsa, nsb):
    """batch_pm_kernel's roles over one CTA's items (chunks per item): loader
    (A slots), builders (B slots), MMA issuer (two accumulators) and epilogue,
    as generators of ('wait', barrier, phase), ('arrive', barrier), ('async',
    barrier) and ('check', barrier, completions needed) ops."""
    def loader():
        gc = 0
        for nch in items:
            for _ in range(nch):
                sl = gc % nsa
                if gc >= nsa:
                    yield ("wait", f"afree{sl}", gc // nsa - 1)
                yield ("check", f"afree{sl}", gc // nsa)  # slot's previous MMAs done
                yield ("async", f"full{sl}")
                gc += 1

    def builders():
        gc = 0
        for nch in items:
            for _ in range(nch):
                sl, bs = gc % nsa, gc % nsb
                yield ("wait", f"full{sl}", gc // nsa)
                if gc >= nsb:
                    yield ("wait", f"bfree{bs}", gc // nsb - 1)
                yield ("check", f"bfree{bs}", gc // nsb)
                yield ("arrive", f"built{bs}")
                gc += 1

    def mma():
        gc = 0
        for it, nch in enumerate(items):
            buf = it & 1
            if it >= 2:
                yield ("wait", f"accempty{buf}", (it >> 1) - 1)
            yield ("check", f"accempty{buf}", it >> 1)  # accumulator read out
            for _ in range(nch):
                sl, bs = gc % nsa, gc % nsb
                yield ("wait", f"full{sl}", gc // nsa)
                yield ("wait", f"built{bs}", gc // nsb)
                yield ("async", f"afree{sl}")
                yield ("async", f"bfree{bs}")
                gc += 1
            yield ("async", f"accfull{buf}")

    def epilogue():
        for it in range(len(items)):
            buf = it & 1
            yield ("wait", f"accfull{buf}", it >> 1)
            yield ("arrive", f"accempty{buf}")

    return [loader(), builders(), mma(), epilogue()]


def test_grouped_point_major_barriers_never_alias_and_never_reuse_early():
    """The same check for the grouped point-major product: over random
    interleavings, every parity wait meets its barrier at most one phase past
    the awaited one, no A slot is refilled and no B slot rebuilt before the
    MMAs of its previous chunk completed, and no item's MMAs start on an
    accumulator before the epilogue read the item two back."""
    rng = random.Random(9)
    for nsa, nsb in ((4, 3), (3, 2), (2, 2), (5, 3)):
        for _ in range(150):
            items = [rng.randint(1, 9) for _ in range(rng.randint(1, 6))]
            roles = _grouped_pm_roles(items, nsa, nsb)
            done, pending = {}, []
            current = [next(r, None) for r in roles]
            while any(c is not None for c in current) or pending:
                choices = [("role", i) for i, c in enumerate(current) if c is not None]
                choices += [("land", i) for i in range(len(pending))]
                kind, i = rng.choice(choices)
                if kind == "land":
                    bar = pending.pop(i)
                    done[bar] = done.get(bar, 0) + 1
                    continue
                op = current[i]
                if op[0] == "wait":
                    completed = done.get(op[1], 0)
                    assert completed <= op[2] + 1, (items, nsa, nsb, op)
                    if completed <= op[2]:
                        assert pending or any(
                            c is not None and not (c[0] == "wait" and done.get(c[1], 0) <= c[2])
                            for c in current), ("stuck", items, current)
                        continue
                elif op[0] == "check":
                    assert done.get(op[1], 0) >= op[2], (items, nsa, nsb, op)
                elif op[0] == "arrive":
                    done[op[1]] = done.get(op[1], 0) + 1
                else:
                    pending.append(op[1])
                current[i] = next(roles[i], None)
