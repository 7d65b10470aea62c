"""Formats the ncu evidence kept in profiles/ (summaries of captures).

  python tr-spmm_b200/trspmm/ncu_summary.py kernel <report.ncu-rep> <algorithmic_bytes>
  python tr-spmm_b200/trspmm/ncu_summary.py launches <launches.csv>

`kernel` prints the figures quoted for one captured launch (duration, DRAM
bytes, throughputs, occupancy, tensor-pipe use) and the per-launch
traffic line that bench.py reads; `launches` prints per-kernel launch counts,
total time and share from a `--metrics gpu__time_duration.sum` launch list.
"""
import csv
import subprocess
import sys

METRICS = [
    ("gpu__time_duration.sum", "duration"),
    ("dram__bytes_read.sum", "dram read"),
    ("dram__bytes_write.sum", "dram write"),
    ("gpu__dram_throughput.avg.pct_of_peak_sustained_elapsed", "dram throughput % of peak"),
    ("lts__throughput.avg.pct_of_peak_sustained_elapsed", "L2 throughput % of peak"),
    ("lts__t_sector_hit_rate.pct", "L2 hit rate %"),
    ("l1tex__throughput.avg.pct_of_peak_sustained_elapsed", "L1 throughput % of peak"),
    ("sm__throughput.avg.pct_of_peak_sustained_elapsed", "SM throughput % of peak"),
    ("sm__pipe_tensor_cycles_active.avg.pct_of_peak_sustained_active", "tensor pipe active %"),
    ("sm__inst_executed_pipe_alu.avg.pct_of_peak_sustained_active", "ALU pipe %"),
    ("sm__inst_executed_pipe_fma.avg.pct_of_peak_sustained_active", "FMA pipe %"),
    ("sm__inst_executed_pipe_lsu.avg.pct_of_peak_sustained_active", "LSU pipe %"),
    ("smsp__inst_executed.sum", "warp instructions"),
    ("sm__warps_active.avg.per_cycle_active", "active warps per SM"),
    ("launch__registers_per_thread", "registers/thread"),
    ("launch__occupancy_limit_registers", "CTA limit (registers)"),
    ("launch__grid_size", "grid"),
]


def _to_bytes(v, unit):
    scale = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}.get(unit)
    return float(v.replace(",", "")) * scale if scale else None


def kernel(rep, algorithmic_bytes=None):
    out = subprocess.run(["ncu", "-i", rep, "--page", "raw", "--csv"], capture_output=True,
                         text=True, check=True).stdout
    rows = list(csv.reader(out.splitlines()))
    hdr, units, vals = rows[0], rows[1], rows[2]
    col = {h: i for i, h in enumerate(hdr)}
    print(f"kernel: {vals[col['Kernel Name']]}")
    traffic = 0.0
    for m, label in METRICS:
        if m in col:
            print(f"  {label:34s} {vals[col[m]]:>16s} {units[col[m]]}")
    for m in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
        traffic += _to_bytes(vals[col[m]], units[col[m]])
    print(f"traffic_bytes_per_launch: {traffic:.0f}")
    if algorithmic_bytes:
        print(f"algorithmic_bytes_per_launch: {float(algorithmic_bytes):.0f}")
        print(f"traffic / algorithmic: {traffic / float(algorithmic_bytes):.2f}")


def launches(path):
    rows = list(csv.reader(open(path)))
    i = [k for k, r in enumerate(rows) if r and r[0] == "ID"][0]
    hdr = rows[i]
    kn, mv = hdr.index("Kernel Name"), hdr.index("Metric Value")
    agg = {}
    for r in rows[i + 1:]:
        if len(r) <= mv or not r[mv].replace(",", "").replace(".", "").isdigit():
            continue
        name = r[kn].split("(")[0]
        a = agg.setdefault(name, [0, 0.0])
        a[0] += 1
        a[1] += float(r[mv].replace(",", ""))
    tot = sum(v[1] for v in agg.values())
    print(f"{'kernel':70s} {'launches':>8s} {'total us':>10s} {'share':>6s}")
    for n, (c, t) in sorted(agg.items(), key=lambda x: -x[1][1]):
        print(f"{n[:70]:70s} {c:8d} {t / 1e3:10.1f} {100 * t / tot:5.1f}%")


if __name__ == "__main__":
    if sys.argv[1] == "kernel":
        kernel(sys.argv[2], sys.argv[3] if len(sys.argv) > 3 else None)
    else:
        launches(sys.argv[2])
