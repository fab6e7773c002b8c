"""Host mirror of the reference's plugin API (src/kernel/mod.rs) over the C ABI.

``KernelTable`` keeps the reference's contract: kernels are keyed by
``(Operator, CpuTarget, MemoryTier)`` (mod.rs:39), ``select`` tries the exact
key for the detected target, then the scalar kernel for the tier, then any
kernel for the operator (mod.rs:209-221), and ``register``/``list`` behave as
mod.rs:229-241. The GPU kernels register under ``CpuTarget.GPU_SM100A`` and
``MemoryTier.HBM``; their ``execute`` calls ``tgp_kernel_execute``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from enum import IntEnum

from . import _capi as A
from .engine import Context


class Operator(IntEnum):
    """src/kernel/mod.rs:48-74 (same order)."""
    ScanEqU64 = 0
    ScanRangeU64 = 1
    ScanMultiPredicate = 2
    HashBuild = 3
    HashProbe = 4
    AggregateSumF64 = 5
    AggregateCountDistinct = 6
    SimilarityHamming = 7
    LeapfrogJoin = 8


class PredicateOp(IntEnum):
    """src/kernel/mod.rs:84-92."""
    Eq = 0
    Gt = 1
    Lt = 2


class MemoryTier(IntEnum):
    """src/memory/tier.rs:11-29."""
    L1L2 = 0
    L3 = 1
    Ddr5 = 2
    Hbm = 3
    Cxl = 4
    Nvme = 5
    NvmeOf = 6
    Network = 7


class CpuTarget(IntEnum):
    """src/kernel/cpu.rs:31-43 plus the GPU target."""
    Scalar = 0
    X86Avx2 = 1
    X86Avx512 = 2
    ArmNeon = 3
    ArmSve = 4
    GpuSm100a = 5


U64_MAX = (1 << 64) - 1


@dataclass
class KernelParams:
    """src/kernel/mod.rs:96-136, defaults as ``impl Default``."""
    target_u64: int = 0
    low_u64: int = 0
    high_u64: int = U64_MAX
    max_distance: int = 0
    cell_count: int = 0
    target2_u64: int = 0
    target3_u64: int = 0
    pred1_op: PredicateOp = PredicateOp.Eq
    pred2_op: PredicateOp = PredicateOp.Eq
    pred3_op: PredicateOp = PredicateOp.Eq
    predicate_count: int = 0

    def to_c(self) -> A.KernelParams:
        p = A.KernelParams()
        p.target_u64, p.low_u64, p.high_u64 = self.target_u64 & U64_MAX, self.low_u64 & U64_MAX, self.high_u64 & U64_MAX
        p.max_distance, p.cell_count = self.max_distance, self.cell_count
        p.target2_u64, p.target3_u64 = self.target2_u64 & U64_MAX, self.target3_u64 & U64_MAX
        p.pred1_op, p.pred2_op, p.pred3_op = int(self.pred1_op), int(self.pred2_op), int(self.pred3_op)
        p.predicate_count = self.predicate_count
        return p


@dataclass
class KernelResult:
    """src/kernel/mod.rs:140-148."""
    count: int = 0
    sum: float = 0.0
    mask: int = 0


class Kernel:
    """``trait Kernel`` (src/kernel/mod.rs:158-177)."""

    def operator(self) -> Operator: raise NotImplementedError
    def cpu(self) -> CpuTarget: raise NotImplementedError
    def tier(self) -> MemoryTier: raise NotImplementedError
    def name(self) -> str: raise NotImplementedError

    def execute(self, input_ptr: int, output_ptr: int | None, params: KernelParams) -> KernelResult:
        raise NotImplementedError


class GpuKernel(Kernel):
    """One sm_100a kernel behind ``tgp_kernel_execute``."""

    def __init__(self, ctx: Context, info: A.KernelInfo):
        self.ctx = ctx
        self._op = Operator(info.op)
        self._cpu = CpuTarget(info.cpu)
        self._tier = MemoryTier(info.tier)
        self._name = info.name.decode()

    def operator(self) -> Operator: return self._op
    def cpu(self) -> CpuTarget: return self._cpu
    def tier(self) -> MemoryTier: return self._tier
    def name(self) -> str: return self._name

    def execute(self, input_ptr: int, output_ptr: int | None, params: KernelParams) -> KernelResult:
        r = self.ctx.kernel_execute(int(self._op), input_ptr, output_ptr, params.to_c())
        return KernelResult(int(r.count), float(r.sum), int(r.mask))


def gpu_kernels(ctx: Context) -> list[GpuKernel]:
    lib = A.load()
    out = []
    for i in range(lib.tgp_kernel_count()):
        info = A.KernelInfo()
        if lib.tgp_kernel_info_at(i, C.byref(info)) != A.OK:
            raise RuntimeError("tgp_kernel_info_at failed")
        out.append(GpuKernel(ctx, info))
    return out


class KernelTable:
    """``struct KernelTable`` (src/kernel/mod.rs:181-242) with the GPU kernels registered."""

    def __init__(self, ctx: Context, detected: CpuTarget = CpuTarget.GpuSm100a):
        self._kernels: dict[tuple[Operator, CpuTarget, MemoryTier], Kernel] = {}
        self._detected = detected
        for k in gpu_kernels(ctx):
            self.register(k)

    def detected_cpu(self) -> CpuTarget:
        return self._detected

    def select(self, op: Operator, tier: MemoryTier) -> Kernel | None:
        k = self._kernels.get((op, self._detected, tier))
        if k is not None:
            return k
        k = self._kernels.get((op, CpuTarget.Scalar, tier))
        if k is not None:
            return k
        for kern in self._kernels.values():
            if kern.operator() == op:
                return kern
        return None

    def register(self, kernel: Kernel) -> None:
        self._kernels[(kernel.operator(), kernel.cpu(), kernel.tier())] = kernel

    def list(self) -> list[tuple[Operator, CpuTarget, MemoryTier, str]]:
        return [(op, cpu, tier, k.name()) for (op, cpu, tier), k in self._kernels.items()]
