"""Shared evaluation of the reference KATs against any backend (oracle or GPU)."""
import numpy as np

from turbogp_b200 import _capi as A
from turbogp_b200.engine import col
from turbogp_b200.kernel_table import KernelParams, Operator, PredicateOp

CMP = {"eq": "__eq__", "ne": "__ne__", "lt": "__lt__", "le": "__le__", "gt": "__gt__", "ge": "__ge__"}


def leaf(name: str, op: str, v):
    return getattr(col(name), CMP[op])(v)


def scalar_expect(values: np.ndarray, op: str, v) -> np.ndarray:
    """The per-row scalar definition the reference's i32 test compares against."""
    x = values.astype(np.int64)
    return {"eq": x == v, "ne": x != v, "lt": x < v, "le": x <= v, "gt": x > v, "ge": x >= v}[op]


def kernel_params(case: dict) -> KernelParams:
    p = case["params"]
    kp = KernelParams()
    if "target_u64" in p:
        kp.target_u64 = p["target_u64"]
    if "low_u64" in p:
        kp.low_u64, kp.high_u64 = p["low_u64"], p["high_u64"]
    if "preds" in p:
        preds = p["preds"]
        kp.predicate_count = len(preds)
        names = [("target_u64", "pred1_op"), ("target2_u64", "pred2_op"), ("target3_u64", "pred3_op")]
        for (t, o), (v, op) in zip(names, preds):
            setattr(kp, t, v)
            setattr(kp, o, PredicateOp[op])
    return kp


def arith_aggs(case: dict):
    """SUM of a sum of products -> one SUM aggregate per product term."""
    from turbogp_b200.engine import Factor, Term, count_star, sum_
    if case.get("count_star"):
        return [count_star()]
    out = []
    for term in case["sum_of"]:
        out.append(sum_(Term([Factor(c, m, a) for c, m, a in term])))
    return out
