"""Cut a small fixture for the ncu_digest tests out of raw-page Nsight Compute CSV exports
(`ncu -i capture.ncu-rep --page raw --csv > capture.csv`): the identification columns and the
metrics the digest groups use, for every launch in each file.

    python tests/golden/make_ncu_sample.py walk.csv infer.csv > tests/golden/ncu_sample.csv
"""

import csv
import re
import sys

KEEP = re.compile(r"^(ID|Kernel Name|gpu__time_duration\.sum|launch__(grid_size|block_size|registers_per_thread)|"
                  r"smsp__issue_active\.avg\.pct_of_peak_sustained_active|"
                  r"smsp__thread_inst_executed_per_inst_executed\.ratio|smsp__inst_executed\.sum|"
                  r"sm__pipe_(alu|fma|tensor)_cycles_active\.avg\.pct_of_peak_sustained_active|"
                  r"sm__inst_executed_pipe_xu\.avg\.pct_of_peak_sustained_active|"
                  r"smsp__average_warps_issue_stalled_(wait|long_scoreboard|not_selected|selected)_per_issue_active\.ratio|"
                  r"l1tex__t_sectors_pipe_lsu_mem_local_op_(ld|st)\.sum|dram__bytes_(read|write)\.sum)$")


def main() -> None:
    tables = []
    for path in sys.argv[1:]:
        rows = [r for r in csv.reader(open(path)) if r]
        tables.append(rows)
    names = [h for h in tables[0][0] if KEEP.match(h)]
    out = csv.writer(sys.stdout, quoting=csv.QUOTE_ALL, lineterminator="\n")
    out.writerow(names)
    idx0 = {h: i for i, h in enumerate(tables[0][0])}
    out.writerow([tables[0][1][idx0[h]] for h in names])
    for rows in tables:
        idx = {h: i for i, h in enumerate(rows[0])}
        for r in rows[2:]:
            out.writerow([r[idx[h]] if h in idx else "" for h in names])


if __name__ == "__main__":
    main()
