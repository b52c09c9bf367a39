"""Comparison of GPU GROUP BY results with the oracle (sorted-set comparison, as the reference's output order is
hash-slot order).  Integer aggregates must match bit for bit; float SUM/AVG within FLOAT_RTOL of the FP64 oracle;
float MIN/MAX exactly (they select an input value)."""
import numpy as np

FLOAT_RTOL = 1e-5  # relative tolerance of float SUM/AVG against the FP64 oracle


def sort_order(keys, key_nulls):
    cols = []
    for k, n in zip(reversed(keys), reversed(key_nulls)):
        cols.append(np.where(n, 0, k))
        cols.append(~n)  # NULL first
    return np.lexsort(cols)


def compare(gpu: dict, ref: dict, aggs, val_is_float: bool, key_is_float: bool = False, rtol: float = FLOAT_RTOL):
    """gpu: GroupByTable.results_numpy(); ref: oracle.groupby(...).  Returns the max relative error of float
    SUM/AVG (0 for integer values)."""
    assert gpu["n_groups"] == ref["count"], f"group count {gpu['n_groups']} != {ref['count']}"
    nk = len(ref["keys"])
    gk = [np.asarray(k, dtype=np.float64 if key_is_float else np.int64) for k in gpu["keys"]]
    gn = [np.asarray(x, dtype=bool) for x in gpu["key_nulls"]]
    order = sort_order(gk, gn)
    for c in range(nk):
        assert (gn[c][order] == ref["key_nulls"][c]).all(), f"key null flags differ in column {c}"
        nn = ~ref["key_nulls"][c]
        assert (gk[c][order][nn] == ref["keys"][c][nn]).all(), f"keys differ in column {c}"
    max_rel = 0.0
    for a in aggs:
        g = np.asarray(gpu[a])[order]
        col = "cnt" if a == "count" else a
        r = ref[col]
        if a == "count":
            assert (g == r).all(), "COUNT differs"
            if a + "_null" in gpu:
                assert not gpu[a + "_null"].any(), "COUNT is never NULL"
            continue
        gnull = gpu[a + "_null"][order]
        assert (gnull == ref["val_null"]).all(), f"{a}: NULL flags differ"
        ok = ~ref["val_null"]
        if val_is_float and a in ("sum", "avg"):
            denom = np.maximum(np.abs(r[ok]), 1e-30)
            rel = np.abs(g[ok].astype(np.float64) - r[ok]) / denom
            if rel.size:
                max_rel = max(max_rel, float(rel.max()))
            assert (rel <= rtol).all(), f"{a}: max relative error {rel.max():.3e} > {rtol}"
        elif val_is_float:
            assert (g[ok].astype(np.float64) == r[ok]).all(), f"{a}: values differ"
        else:
            assert (g[ok].astype(np.int64) == r[ok]).all(), f"{a}: values differ"
    return max_rel
