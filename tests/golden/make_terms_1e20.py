"""Per-term values of the Deleglise-Rivat decomposition at x = 10^20, y = 16 *
icbrt(x) = 74265408, c = 6, from the CPU oracle (oracle/oracle.c): P2 by
pi-table windows over [sqrt x, z] (z = 1346521923100), ordinary, trivial and
pi(y).  Writes terms_1e20.json beside this script; about half an hour on 8
cores.

The total pi(10^20) = 2220819602560918840 (OEIS A006880) is in golden.json; the
GPU test checks P2, ordinary, trivial and pi(y) against this file and the total
against OEIS."""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402


def main():
    x = 10**20
    y = 16 * oracle.icbrt(x)
    out = {"x": str(x), "y": y, "c": 6}
    t = time.time()
    out["ordinary"] = str(oracle.ordinary(x, y, 6))
    out["trivial"] = str(oracle.trivial(x, y))
    out["pi_y"] = str(oracle.pi_sieve(y))
    print("ordinary/trivial/pi_y", out, round(time.time() - t, 1), flush=True)
    out["P2"] = str(oracle.P2(x, y))
    out["seconds"] = round(time.time() - t, 1)
    with open(os.path.join(HERE, "terms_1e20.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out, flush=True)


if __name__ == "__main__":
    main()
