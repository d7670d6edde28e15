"""One rank of the two-process bench test: joins a gloo group on 127.0.0.1 and
prints what bench.py's cross-rank helpers return on it (test infrastructure)."""
import datetime
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    rank, world, port = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=port)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    local = [3.0, 5.0, 4.0, 1.0][rank]          # this rank's elapsed seconds
    slowest = bench.max_over_ranks(local, world, "cpu")
    value = bench.replica_throughput(1000, world, slowest)
    dist.barrier()
    dist.destroy_process_group()
    print(json.dumps({"rank": rank, "slowest": slowest, "value": value}))


if __name__ == "__main__":
    main()
