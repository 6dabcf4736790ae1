"""Bank model of the FP64 line-thread stage buffers (csrc/hex27.cuh H27Fp64Banked and the
slot strides of the kernels that use it), recomputed from the constants in the sources.

A warp holds three elements of nine line threads (lanes 0..26) and five idle lanes; an FP64
shared-memory access is served as two half-warps of 16 lanes over 16 eight-byte banks, and
a half-warp takes as many wavefronts as the largest number of distinct words that share a
bank. One gradient (h27_gradient) and one transpose (h27_transpose) access their two buffer
kinds in three line orientations; the counts below are per gradient + transpose and lane
group, against the floor of two wavefronts per access (384). CPU only."""
import os
import re

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "femtools.jl_b200", "csrc")

# (orientation, buffer kind, accesses per gradient + transpose, is a store)
ACCESSES = [("A", 1, 18, True), ("B", 1, 18, False), ("B", 2, 27, True), ("C", 2, 27, False),
            ("C", 2, 30, True), ("B", 2, 30, False), ("B", 1, 21, True), ("A", 1, 21, False)]


def src(name):
    with open(os.path.join(CSRC, name)) as f:
        return f.read()


def banked_layout():
    s = src("hex27.cuh")
    body = s[s.index("struct H27Fp64Banked"):]
    body = body[:body.index("};")]
    k1, k2 = map(int, re.search(r"K1 = (\d+), K2 = (\d+)", body).groups())
    slot, idle = map(int, re.search(r"SLOT = (\d+), IDLE_M = (\d+)", body).groups())
    l1 = tuple(map(int, re.search(r"l1\(int i, int j, int k\) \{ return (\d+) \* i \+ (\d+) \* j \+ (\d+) \* k", body).groups()))
    l2 = tuple(map(int, re.search(r"l2\(int i, int j, int k\) \{ return (\d+) \* i \+ (\d+) \* j \+ (\d+) \* k", body).groups()))
    return dict(K1=k1, K2=k2, SLOT=slot, IDLE_M=idle, l1=l1, l2=l2)


def wavefronts(addr):
    total = 0
    for half in (addr[:16], addr[16:]):
        banks = {}
        for w in half:
            if w is not None:
                banks.setdefault(w % 16, set()).add(w)
        total += max(len(v) for v in banks.values())
    return total


def cost(l1, l2, stride, idle_slot, idle_m, idle_writes=True):
    def form(kind, a, b, c):
        return {"A": lambda m1, m2: b * m1 + c * m2, "B": lambda m1, m2: a * m1 + c * m2,
                "C": lambda m1, m2: a * m1 + b * m2}[kind]
    total = 0
    for kind, buf, n, store in ACCESSES:
        f = form(kind, *(l1 if buf == 1 else l2))
        addr = []
        for lane in range(32):
            if lane < 27:
                s, m = lane // 9, lane % 9
            elif store and not idle_writes:
                addr.append(None)
                continue
            else:
                s, m = idle_slot, idle_m
            addr.append(s * stride + f(m % 3, m // 3))
        total += n * wavefronts(addr)
    return total


def test_layouts_are_one_to_one_within_their_blocks():
    L = banked_layout()
    for coef, K in ((L["l1"], L["K1"]), (L["l2"], L["K2"])):
        vals = {coef[0] * i + coef[1] * j + coef[2] * k for i in range(3) for j in range(3) for k in range(3)}
        assert len(vals) == 27 and max(vals) < K
    # a gradient's two buffers and a transpose's two buffers fit one slot
    assert max(6 * L["K1"] + 9 * L["K2"], 10 * L["K2"] + 7 * L["K1"]) <= L["SLOT"]


def test_four_slot_kernels():
    # general residual, adjoint, cell pressure: slots SLOT words apart, idle lanes in slot 3
    L = banked_layout()
    assert cost(L["l1"], L["l2"], L["SLOT"], 3, L["IDLE_M"]) == 480
    assert cost((1, 3, 9), (1, 3, 9), 540, 3, 0) == 807          # the compact layout
    assert "LY::SLOT" in src("cellpressure.cu") and "H27Layout<T>" in src("stokes3d.cu")


def test_pipelined_and_jacobian_strides():
    L = banked_layout()
    pipe = src("stokes3d_pipe.cu")
    words, idle_s, idle_m = map(int, re.search(
        r"struct PipeStage<double> \{\s*using LY = H27Fp64Banked;\s*static constexpr int WORDS = (\d+), IDLE_S = (\d+), "
        r"IDLE_M = (\d+);", pipe).groups())
    # idle lanes read but never write in the pipelined kernel
    assert cost(L["l1"], L["l2"], words, idle_s, idle_m, idle_writes=False) == 480
    assert cost((1, 3, 9), (1, 3, 9), 500, 0, 0, idle_writes=False) == 750
    jac = src("jacobian3d.cu")
    e_stride = int(re.search(r"e_stride = strided \? 1025 : (\d+);", jac).group(1))
    assert cost(L["l1"], L["l2"], e_stride, 3, L["IDLE_M"]) == 480
    assert cost((1, 3, 9), (1, 3, 9), 864, 3, 8) == 1152
