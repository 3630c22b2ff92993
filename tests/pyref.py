"""Independent pure-Python restatement of SIGMo's hot path, for small inputs.

Written separately from the C++ oracle (oracle/sigmo_oracle.cpp) so the two
can check each other; used by tests/golden/make_golden.py to produce the
committed golden vectors.  Each function follows the reference file:line it
names.  Profiles: 0 REF_PTX, 1 REF_X86, 2 EXACT.
"""
from __future__ import annotations

REF_PTX, REF_X86, EXACT = 0, 1, 2
M32, M64 = (1 << 32) - 1, (1 << 64) - 1


def _shl64_one(count: int, prof: int) -> int:
    if prof == REF_X86:
        return 1 << (count & 63)
    return 0 if count >= 64 else 1 << count


def _shl32(v: int, c: int, prof: int) -> int:
    if prof == REF_X86:
        return (v << (c & 31)) & M32
    return 0 if c >= 32 else (v << c) & M32


def _shr32(v: int, c: int, prof: int) -> int:
    if prof == REF_X86:
        return v >> (c & 31)
    return 0 if c >= 32 else v >> c


# Signature word (signature.hpp:23-54)
def sig_get(s: int, label: int) -> int:
    label &= 0xFF
    return (s >> (label * 4)) & 0xF if label < 16 else 0


def sig_set(s: int, label: int, count: int) -> int:
    label &= 0xFF
    count &= 0xFF
    if label < 16 and count < 16:
        s &= ~(0xF << (label * 4)) & M64
        s |= count << (label * 4)
    return s


def sig_inc(s: int, label: int, add: int = 1) -> int:
    label &= 0xFF
    if label < 16:
        c = sig_get(s, label)
        if c < 15:
            s = sig_set(s, label, (c + add) & 0xFF)
    return s


class Bitset:
    """utils::detail::Bitset<uint64_t> (utils.hpp:64-96)."""

    def __init__(self, offset: int, prof: int):
        self.data, self.offset, self.prof = 0, offset, prof

    def _c(self, idx):
        return ((idx & 0xFF) - self.offset) & M32

    def set(self, idx):
        self.data |= _shl64_one(self._c(idx), self.prof)

    def unset(self, idx):
        self.data &= ~_shl64_one(self._c(idx), self.prof) & M64

    def get(self, idx):
        return (self.data & _shl64_one(self._c(idx), self.prof)) != 0

    def set_bits(self):
        return [b for b in range(64) if (self.data >> b) & 1]


def graph_id(goff, v):
    """getGraphID (graph.hpp:100-111)."""
    lo, hi = 0, len(goff) - 1
    while lo < hi:
        mid = (lo + hi) // 2
        if v >= goff[mid]:
            lo = mid + 1
        else:
            hi = mid
    return lo - 1


def generate_signatures(g, sig):
    """generateCSRSignatures (signature.hpp:125-152)."""
    ro, col, lab = g["row_offsets"], g["column_indices"], g["node_labels"]
    for v in range(len(lab)):
        for i in range(ro[v], ro[v + 1]):
            sig[v] = sig_inc(sig[v], lab[col[i]])
    return sig


def refine_signatures(g, view, prof, sig, reach):
    """refineCSRSignatures<PowerGraph> (signature.hpp:336-390); reach: list of
    python ints (bitsets of arbitrary width under EXACT)."""
    goff, ro, col, lab = g["graph_offsets"], g["row_offsets"], g["column_indices"], g["node_labels"]
    for v in range(len(lab)):
        prev = goff[graph_id(goff, v)]
        if prof != EXACT:
            fr, re = Bitset(0, prof), Bitset(0, prof)
            fr.set(v - prev)
            re.set(v - prev)
            it = 0
            while it < view and fr.data:
                nx = Bitset(0, prof)
                for b in fr.set_bits():
                    u = b + prev
                    for i in range(ro[u], ro[u + 1]):
                        nb = col[i] - prev
                        if not re.get(nb):
                            re.set(nb)
                            nx.set(nb)
                fr = nx
                it += 1
            re.unset(v - prev)
            sphere = re.data & ~reach[v] & M64
            s = 0
            for b in range(64):
                if (sphere >> b) & 1:
                    s = sig_inc(s, lab[prev + b])
            sig[v] = s
            reach[v] = sphere | reach[v]
        else:
            lv = v - prev
            fr, re = {lv}, {lv}
            for _ in range(view):
                if not fr:
                    break
                nx = set()
                for u in fr:
                    for i in range(ro[u + prev], ro[u + prev + 1]):
                        nb = col[i] - prev
                        if nb not in re:
                            re.add(nb)
                            nx.add(nb)
                fr = nx
            re.discard(lv)
            old = reach[v]
            s = 0
            newbits = 0
            for b in sorted(re):
                if not (old >> b) & 1:
                    s = sig_inc(s, lab[prev + b])
                newbits |= 1 << b
            sig[v] = s
            reach[v] = old | newbits
    return sig


def words(n):
    return (n + 31) // 32


def filter_candidates(q, d):
    """filterCandidates<Query> (isomorphism.hpp:22-62); bits[q] = python int row."""
    ql, dl = q["node_labels"], d["node_labels"]
    rows = []
    for a in ql:
        r = 0
        for j, b in enumerate(dl):
            if a == b or a == 255:
                r |= 1 << j
        rows.append(r)
    return rows


def refine_candidates(q, d, sq, sd, rows):
    """refineCandidates<Query> race-free (isomorphism.hpp:64-127)."""
    out = []
    for qi, r in enumerate(rows):
        nr = 0
        for j in range(len(d["node_labels"])):
            if (r >> j) & 1 and all(sig_get(sq[qi], l) <= sig_get(sd[j], l) for l in range(16)):
                nr |= 1 << j
        out.append(nr)
    return out


def _word(row, i):
    return (row >> (32 * i)) & M32


def _mask(i, s, e, prof):
    si, ei = s // 32, (e + 31) // 32
    if prof == EXACT:
        lo, hi = max(s, 32 * i), min(e, 32 * i + 32)
        if lo >= hi:
            return 0
        return (((1 << (hi - lo)) - 1) << (lo - 32 * i)) & M32
    m = M32
    if si == ei - 1:
        m = _shl32(_shr32(m, (32 - (e - s)) & M32, prof), s % 32, prof)
    elif i == si:
        m = _shl32(m, s % 32, prof)
    elif i == ei - 1:
        m = _shr32(m, (32 - e % 32) & M32, prof)
    return m


def cand_list(row, s, e, prof):
    """getCandidateAt for every index (candidates.hpp:132-162)."""
    out = []
    for i in range(s // 32, (e + 31) // 32):
        blk = _word(row, i) & _mask(i, s, e, prof)
        for t in range(32):
            if (blk >> t) & 1:
                out.append(32 * i + t)
    return out


def gmcr(q, d, rows, prof):
    """generateGMCR (gmcr.hpp:33-128), sorted segments, <=1-vertex queries skipped."""
    qg, dg = q["graph_offsets"], d["graph_offsets"]
    offsets, indices = [0], []
    for g in range(len(dg) - 1):
        s, e = dg[g], dg[g + 1]
        for qi in range(len(qg) - 1):
            n = qg[qi + 1] - qg[qi]
            if n <= 1:
                continue
            if all(cand_list(rows[qg[qi] + j], s, e, prof) for j in range(n)):
                indices.append(qi)
        offsets.append(len(indices))
    return offsets, indices


def _nb(g, a, b):
    ro, col = g["row_offsets"], g["column_indices"]
    return any(col[i] == b for i in range(ro[a], ro[a + 1]))


def join(q, d, rows, offsets, indices, prof, find_first, wg=128):
    """joinCandidates (isomorphism.hpp:270-381), literal DFS per simulated item."""
    qg, dg = q["graph_offsets"], d["graph_offsets"]
    per = [0] * len(indices)
    for g in range(len(dg) - 1):
        s, e = dg[g], dg[g + 1]
        seg0, seglen = offsets[g], offsets[g + 1] - offsets[g]
        for lid in range(min(wg, seglen)):
            mapping = [0] * 65
            for it in range(lid, seglen, wg):
                qi = indices[seg0 + it]
                qoff, n = qg[qi], qg[qi + 1] - qg[qi]
                cands = [cand_list(rows[qoff + j], s, e, prof) for j in range(n)]
                found = 0
                stack = [[0, 0]]
                if prof != EXACT:
                    vis = Bitset(s, prof)
                    while stack:
                        depth, idx = stack[-1]
                        if depth == n:
                            found += 1
                            stack.pop()
                            if find_first:
                                break
                            continue
                        if idx >= len(cands[depth]):
                            stack.pop()
                            vis.unset(mapping[depth])
                            if len(stack) == 1:
                                vis.data = 0
                            continue
                        c = cands[depth][idx]
                        stack[-1][1] += 1
                        if vis.get(c):
                            continue
                        if depth == 0 or all(_nb(q, i + qoff, depth + qoff) == _nb(d, mapping[i], c) for i in range(depth)):
                            mapping[depth] = c
                            vis.set(c)
                            stack.append([depth + 1, 0])
                else:
                    # injective DFS (recursive)
                    m = [0] * n

                    def rec(depth, used):
                        if depth == n:
                            return 1
                        tot = 0
                        for c in cands[depth]:
                            if c in used:
                                continue
                            if all(_nb(q, i + qoff, depth + qoff) == _nb(d, m[i], c) for i in range(depth)):
                                m[depth] = c
                                tot += rec(depth + 1, used | {c})
                                if find_first and tot:
                                    return tot
                        return tot

                    found = rec(0, frozenset())
                    if find_first:
                        found = min(found, 1)
                per[seg0 + it] = found
    return sum(per), per


def as_lists(b):
    return {k: [int(x) for x in getattr(b, k)] for k in
            ("graph_offsets", "row_offsets", "column_indices", "node_labels", "edge_labels")}


def run_pipeline(qb, db, iterations, prof, find_first, wg=128):
    q, d = as_lists(qb), as_lists(db)
    sd = generate_signatures(d, [0] * len(d["node_labels"]))
    sq = generate_signatures(q, [0] * len(q["node_labels"]))
    rows = filter_candidates(q, d)
    hist = {"bitsets": [list(rows)], "sig_data": [list(sd)], "sig_query": [list(sq)]}
    rd, rq = [0] * len(sd), [0] * len(sq)
    for r in range(1, iterations + 1):
        refine_signatures(d, r, prof, sd, rd)
        refine_signatures(q, r, prof, sq, rq)
        rows = refine_candidates(q, d, sq, sd, rows)
        hist["bitsets"].append(list(rows))
        hist["sig_data"].append(list(sd))
        hist["sig_query"].append(list(sq))
    offsets, indices = gmcr(q, d, rows, prof)
    total, per = join(q, d, rows, offsets, indices, prof, find_first, wg)
    hist.update(offsets=offsets, indices=indices, total=total, per_pair=per)
    return hist


def rows_to_words(rows, n):
    """python-int rows -> list of lists of uint32 words (reference layout)."""
    W = words(n)
    return [[(r >> (32 * i)) & M32 for i in range(W)] for r in rows]
