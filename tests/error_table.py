"""Summarise the per-case maximum errors that the GPU parity tests append to
$SRK_ERROR_LOG (tests/windows.py ErrorLog) as a markdown table:

    SRK_ERROR_LOG=errors.jsonl python -m pytest tests/test_gpu_configs.py -m gpu
    python tests/error_table.py errors.jsonl
"""
import json
import sys


def main(path):
    rows = {}
    with open(path) as fh:
        for line in fh:
            r = json.loads(line)
            key = (r["op"], r["N"], r["KW"], r["dtype"])
            old = rows.get(key)
            if old is None or r["windows"] > old["windows"] or (r["windows"] == old["windows"] and r["max_rel"] > old["max_rel"]):
                rows[key] = r
    print("| op | N | KW | storage | windows x pixels | max abs err / max abs ref | pixels outside the per-pixel rule |")
    print("|---|---|---|---|---|---|---|")
    for (op, N, KW, dt) in sorted(rows):
        r = rows[(op, N, KW, dt)]
        per = r["pixels"] // max(r["windows"], 1)
        win = "%d x %d^2" % (r["windows"], int(round(per ** 0.5))) if r["windows"] else "dot product"
        print("| %s | %d | %d | %s | %s | %.2e | %d |" % (op, N, KW, dt, win, r["max_rel"], r["pixel_violations"]))


if __name__ == "__main__":
    main(sys.argv[1])
