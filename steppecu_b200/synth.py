"""Seeded synthetic PACKEDANCESTRYMAP panels with the shapes of the f2 extraction workloads.

No public dataset is available offline, so panels are drawn from a Balding-Nichols model:
ancestral frequency p ~ U(0.05, 0.95) per SNP, population frequency
Beta(p(1-F)/F, (1-p)(1-F)/F), diploid genotype Binomial(2, p_pop), pseudo-haploid one
allele coded 0 or 2, missing code 3. Individuals are interleaved across populations in
file order (as in real panels), so selecting a population is a gather. Genetic positions
are physical positions at 1 cM/Mb; the jackknife blocks follow the AT2 walk.

Generation uses torch on any device (CUDA for the large panels); a panel is a pure
function of (workload, seed, device type).
"""
from __future__ import annotations

import dataclasses
import math
from pathlib import Path

import numpy as np
import torch

from .blocks import assign_blocks

# Human-like autosomal genetic lengths (cM), 22 chromosomes, ~3,520 cM in total.
HUMAN_CM = [278, 263, 224, 213, 204, 193, 187, 170, 168, 173, 160, 168, 126, 119, 141, 134, 128,
            126, 107, 108, 62, 72]


@dataclasses.dataclass
class Workload:
    name: str
    n_pop: int
    ind_per_pop: int | None          # None -> lognormal sizes
    n_snp: int
    chrom_cm: list[float]
    missing: str                     # "iid5" | "beta23"
    pseudo_haploid_frac: float
    f_range: tuple[float, float]
    blgsize: float = 0.05            # Morgans
    block_sizes_lognormal: bool = False


WORKLOADS = {
    # 20 pops x 20 diploid, 50k SNPs on 2 chromosomes, 5 cM blocks (~40), F = 0.05, 5% iid missing
    "c1": Workload("c1", 20, 20, 50_000, [100.0, 100.0], "iid5", 0.0, (0.05, 0.05)),
    # 100 pops x 20 (half pseudo-haploid), 1.15M SNPs on 22 chromosomes, per-sample missing ~ Beta(2,3)
    "c2": Workload("c2", 100, 20, 1_150_000, HUMAN_CM, "beta23", 0.5, (0.01, 0.15)),
    # 1000 pops x 10, same SNP/block layout and sample model as c2
    "c3": Workload("c3", 1000, 10, 1_150_000, HUMAN_CM, "beta23", 0.5, (0.01, 0.15)),
    # 1000 pops of lognormal size (1-60), lognormal block sizes (median 1500, 50-6000)
    "c4": Workload("c4", 1000, None, 1_150_000, HUMAN_CM, "beta23", 0.5, (0.01, 0.15),
                   block_sizes_lognormal=True),
    # The shared panel of the many-requests workload: 8,000 samples (400 pops x 20), 1.15M
    # SNPs, same sample model as c2; requests come from batch_requests().
    "c5": Workload("c5", 400, 20, 1_150_000, HUMAN_CM, "beta23", 0.5, (0.01, 0.15)),
}


@dataclasses.dataclass
class Panel:
    records: torch.Tensor       # [n_snp, bytes_per_record] uint8, SNP-major PACKEDANCESTRYMAP
    n_ind: int
    n_snp: int
    bytes_per_record: int
    chrom: np.ndarray           # int32 [n_snp]
    physpos: np.ndarray         # float64 [n_snp]
    genpos: np.ndarray          # float64 [n_snp], Morgans
    ind_pop: np.ndarray         # int32 [n_ind]: population index of each file row
    pop_labels: list[str]
    ploidy_true: np.ndarray     # int32 [n_ind]: 2 diploid, 1 pseudo-haploid (generator truth)
    block_id: np.ndarray        # int32 [n_snp]
    n_block: int

    @property
    def n_pop(self) -> int:
        return len(self.pop_labels)

    def selection(self, pops: list[int] | None = None) -> tuple[np.ndarray, np.ndarray]:
        """(sel_rows, pop_offsets) for the given population indices (default: all), in the
        given order; within a population, file order (io::GenoReader::build_selection)."""
        pops = list(range(self.n_pop)) if pops is None else list(pops)
        order = np.argsort(self.ind_pop, kind="stable")
        counts = np.bincount(self.ind_pop, minlength=self.n_pop)
        starts = np.concatenate([[0], np.cumsum(counts)])
        rows, offs = [], [0]
        for p in pops:
            r = order[starts[p]:starts[p + 1]]
            rows.append(r)
            offs.append(offs[-1] + len(r))
        sel = np.concatenate(rows).astype(np.int64) if rows else np.zeros(0, np.int64)
        return sel, np.asarray(offs, dtype=np.int64)

    def records_numpy(self) -> np.ndarray:
        return self.records.cpu().numpy()


def _positions(wl: Workload, rng: np.random.Generator, n_snp: int):
    lens = np.asarray(wl.chrom_cm, dtype=np.float64)
    per = np.floor(n_snp * lens / lens.sum()).astype(np.int64)
    per[: n_snp - per.sum()] += 1
    chrom, phys = [], []
    for c, (L, k) in enumerate(zip(lens, per), start=1):
        pos = np.sort(rng.integers(1, int(L * 1e6), size=k)).astype(np.float64)
        chrom.append(np.full(k, c, np.int32))
        phys.append(pos)
    chrom = np.concatenate(chrom)
    phys = np.concatenate(phys)
    return chrom, phys, phys * 1e-8


def _lognormal_blocks(rng: np.random.Generator, n_snp: int) -> np.ndarray:
    sizes = []
    total = 0
    while total < n_snp:
        k = int(np.clip(round(1500 * math.exp(rng.normal(0.0, 0.8))), 50, 6000))
        k = min(k, n_snp - total)
        sizes.append(k)
        total += k
    return np.repeat(np.arange(len(sizes), dtype=np.int32), sizes)


def _pack(codes: torch.Tensor, bpr: int) -> torch.Tensor:
    """codes [m, N] uint8 in {0,1,2,3} -> PA records [m, bpr], 4 codes per byte MSB-first."""
    m, n = codes.shape
    pad = (-n) % 4
    if pad:
        codes = torch.cat([codes, torch.zeros(m, pad, dtype=torch.uint8, device=codes.device)], dim=1)
    c = codes.view(m, -1, 4).to(torch.int32)
    packed = ((c[:, :, 0] << 6) | (c[:, :, 1] << 4) | (c[:, :, 2] << 2) | c[:, :, 3]).to(torch.uint8)
    if packed.shape[1] < bpr:
        packed = torch.cat([packed, torch.zeros(m, bpr - packed.shape[1], dtype=torch.uint8,
                                                device=codes.device)], dim=1)
    return packed.contiguous()


def generate(workload: str | Workload, seed: int = 20261203, device: str | torch.device = "cpu",
             n_snp: int | None = None, n_pop: int | None = None, chunk: int = 1 << 15) -> Panel:
    """Draws a panel. n_snp / n_pop override the workload's sizes (for small test cases)."""
    wl = WORKLOADS[workload] if isinstance(workload, str) else workload
    M = wl.n_snp if n_snp is None else n_snp
    P = wl.n_pop if n_pop is None else n_pop
    rng = np.random.default_rng(seed)
    device = torch.device(device)

    if wl.ind_per_pop is None:
        sizes = np.clip(np.round(10.0 * np.exp(rng.normal(0.0, 0.7, size=P))), 1, 60).astype(np.int64)
    else:
        sizes = np.full(P, wl.ind_per_pop, np.int64)
    ind_pop = np.repeat(np.arange(P, dtype=np.int32), sizes)
    rng.shuffle(ind_pop)  # interleave populations in file order
    N = int(ind_pop.size)
    ploidy = np.where(rng.random(N) < wl.pseudo_haploid_frac, 1, 2).astype(np.int32)
    if wl.missing == "iid5":
        miss = np.full(N, 0.05)
    else:
        miss = rng.beta(2.0, 3.0, size=N)
    F = rng.uniform(wl.f_range[0], wl.f_range[1], size=P)
    chrom, phys, gen = _positions(wl, rng, M)
    if wl.block_sizes_lognormal:
        block_id = _lognormal_blocks(rng, M)
        n_block = int(block_id[-1]) + 1 if M else 0
    else:
        block_id, n_block = assign_blocks(chrom, gen, wl.blgsize, phys)

    bpr = max(48, (N + 3) // 4)
    out = torch.empty((M, bpr), dtype=torch.uint8, device=device)
    gen_t = torch.Generator(device=device)
    gen_t.manual_seed(seed)
    torch.manual_seed(seed)
    Ft = torch.as_tensor(F, dtype=torch.float32, device=device)[:, None]
    popt = torch.as_tensor(ind_pop, dtype=torch.int64, device=device)
    dip = torch.as_tensor(ploidy == 2, device=device)[None, :]
    missp = torch.as_tensor(miss, dtype=torch.float32, device=device)[None, :]
    for s0 in range(0, M, chunk):
        m = min(chunk, M - s0)
        p_anc = 0.05 + 0.9 * torch.rand(m, generator=gen_t, device=device)
        a = (p_anc[None, :] * (1 - Ft) / Ft).clamp_min(1e-6)
        b = ((1 - p_anc[None, :]) * (1 - Ft) / Ft).clamp_min(1e-6)
        x = torch._standard_gamma(a)
        y = torch._standard_gamma(b)
        p_pop = (x / (x + y)).nan_to_num(0.5)                       # [P, m]
        p_ind = p_pop.index_select(0, popt).t()                     # [m, N]
        a1 = torch.rand(p_ind.shape, generator=gen_t, device=device) < p_ind
        a2 = torch.rand(p_ind.shape, generator=gen_t, device=device) < p_ind
        code = torch.where(dip, a1.to(torch.uint8) + a2.to(torch.uint8), 2 * a1.to(torch.uint8))
        gone = torch.rand(p_ind.shape, generator=gen_t, device=device) < missp
        code = torch.where(gone, torch.full_like(code, 3), code)
        out[s0:s0 + m] = _pack(code, bpr)
        del p_anc, a, b, x, y, p_pop, p_ind, a1, a2, code, gone
    labels = [f"pop{i:04d}" for i in range(P)]
    return Panel(out, N, M, bpr, chrom, phys, gen, ind_pop, labels, ploidy, block_id, n_block)


def write_eigenstrat(panel: Panel, prefix: str | Path) -> None:
    """Writes <prefix>.geno (PACKEDANCESTRYMAP), .snp and .ind."""
    prefix = str(prefix)
    bpr = panel.bytes_per_record
    head = f"GENO {panel.n_ind} {panel.n_snp} 0 0".encode()
    head = head + b"\0" * (bpr - len(head))
    with open(prefix + ".geno", "wb") as f:
        f.write(head)
        f.write(panel.records_numpy().tobytes())
    with open(prefix + ".snp", "w") as f:
        for s in range(panel.n_snp):
            f.write(f"rs{s} {panel.chrom[s]} {panel.genpos[s]:.10f} {int(panel.physpos[s])} A C\n")
    with open(prefix + ".ind", "w") as f:
        for g in range(panel.n_ind):
            f.write(f"I{g} U {panel.pop_labels[panel.ind_pop[g]]}\n")


def batch_requests(panel: Panel, n_req: int = 64, seed: int = 20261208, p_min: int = 4, p_max: int = 300,
                   blgsize: float = 0.05) -> list[dict]:
    """Independent extraction requests over one panel: each selects P_r populations, P_r
    log-uniform on [p_min, p_max], a random subset in ascending order, and has its own 5 cM
    block map (the panel's genetic map scaled by a per-request factor in [0.9, 1.1], i.e. a
    different recombination map, then the AT2 block walk)."""
    rng = np.random.default_rng(seed)
    p_max = min(p_max, panel.n_pop)
    out = []
    for _ in range(n_req):
        P = int(round(math.exp(rng.uniform(math.log(p_min), math.log(p_max)))))
        P = max(1, min(P, panel.n_pop))
        pops = np.sort(rng.choice(panel.n_pop, size=P, replace=False)).tolist()
        sel, po = panel.selection(pops)
        scale = rng.uniform(0.9, 1.1)
        bid, nb = assign_blocks(panel.chrom, panel.genpos * scale, blgsize, panel.physpos)
        out.append({"pops": pops, "sel_rows": sel, "pop_offsets": po, "block_id": np.asarray(bid, np.int32),
                    "n_block": int(nb)})
    return out
