"""One plain solve of the benchmark network, for profiler captures.

``python -m andfn_b200.profile_run [MAX_ITERATIONS]`` builds the same seeded
2,118-fracture network as bench.py and solves it once through the C ABI.
"""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    import bench

    import andfn_b200
    F, E = bench.build_network()
    c = bench.constants()
    if len(sys.argv) > 1:
        c["MAX_ITERATIONS"] = int(sys.argv[1])
    andfn_b200.solve(F, E, 50, c)
    st = andfn_b200.last_stats
    print(f"iterations {st['iterations']} status {st['status']} factor {st['ms_factor']:.1f} ms "
          f"iterate {st['ms_iterate']:.1f} ms")


if __name__ == "__main__":
    main()
