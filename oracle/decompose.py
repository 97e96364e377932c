"""Oracle for the out-of-core decomposition -- TEST INFRASTRUCTURE ONLY.

Restates talshTensorOpDecompose2 (talshc.cpp:3150-3294), the reference's rule
for halving a tensor contraction, in plain Python, and the driver loop of
talshTensorContractXL (talshc.cpp:5507-5551: every operation that is still too
large is replaced by its two children, in order, until none is).  The stop
condition is the one talsh-b200 uses -- the D, L and R blocks of a piece fit a
quarter of the free device budget -- instead of the reference's device-buffer
test (its buddy allocator has no counterpart here); the split choice is the
reference's.  Only tests/ import this module.
"""


def decompose2(cptrn, drank, lrank, rrank, block):
    """One halving.  block = (offsets, extents) with offsets/extents a triple of
    lists for D, L, R.  Returns the two children or None when nothing splits."""
    offs, dims = block
    ldims, rdims = dims[1], dims[2]
    lc = ll = lr = lb = 1
    sc = sl = sr = sb = 0
    mc = ml = mr = mb = -1
    dst = [0] * drank
    for i in range(lrank):  # talshc.cpp:3179-3189
        cd = ldims[i]
        if cptrn[i] < 0:
            lc *= cd
            if cd >= sc:
                sc, mc = cd, i
        elif cptrn[i] > 0:
            dst[cptrn[i] - 1] = i + 1
            ll *= cd
            if cd >= sl:
                sl, ml = cd, i
    for i in range(rrank):  # :3190-3200
        cd = rdims[i]
        j = cptrn[lrank + i]
        if j > 0:
            if dst[j - 1] == 0:
                lr *= cd
                if cd >= sr:
                    sr, mr = cd, lrank + i
            else:  # batch (hyper) index
                ll //= cd
                lb *= cd
                if cd >= sb:
                    sb, mb = cd, lrank + i
    if not (lb > 1 or lr > 1 or ll > 1 or lc > 1):
        return None
    d0 = d1 = d2 = -1  # :3202-3216
    if lb > 1:
        d0 = cptrn[mb] - 1
        d1 = dst[d0] - 1
        d2 = mb - lrank
    elif lr >= ll and lr >= lc:
        d0 = cptrn[mr] - 1
        d2 = mr - lrank
    elif ll >= lr and ll >= lc:
        d0 = cptrn[ml] - 1
        d1 = ml
    else:
        d1 = mc
        d2 = -cptrn[mc] - 1
    c1 = ([list(x) for x in offs], [list(x) for x in dims])
    c2 = ([list(x) for x in offs], [list(x) for x in dims])
    for a, x in enumerate((d0, d1, d2)):  # halves: ceil(n/2) then the rest, :3218-3270
        if x < 0:
            continue
        h1 = (dims[a][x] + 1) // 2
        h2 = dims[a][x] - h1
        if h2 <= 0:
            return None
        c1[1][a][x] = h1
        c2[1][a][x] = h2
        c2[0][a][x] += h1
    return c1, c2


def xl_plan(cptrn, ddims, ldims, rdims, esize, budget_bytes, max_ops=1 << 16):
    """The pieces of an out-of-core contraction, in execution order."""
    ranks = (len(ddims), len(ldims), len(rdims))

    def nbytes(dims):
        v = esize
        for x in dims:
            v *= x
        return v

    ops = [([[0] * r for r in ranks], [list(ddims), list(ldims), list(rdims)])]
    again = True
    while again:
        again = False
        nxt = []
        for b in ops:
            need = sum(nbytes(d) for d in b[1])
            kids = decompose2(cptrn, *ranks, b) if need * 4 > budget_bytes else None
            if kids:
                nxt.extend(kids)
                again = True
            else:
                nxt.append(b)
        ops = nxt
        if len(ops) > max_ops:
            return None
    return ops
