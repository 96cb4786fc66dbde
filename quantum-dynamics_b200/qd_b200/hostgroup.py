"""Host-side rank group of one node: barrier, all-gather and max over the
processes of a job, through files in a directory they share.

The propagations of a batch exchange nothing while they step (replicas), so
the only collective steps a sharded job takes are one gather of per-run
results at the end and, in a benchmark, a barrier and the max of the ranks'
device times.  Those need no device library: every rank writes its value to
`<dir>/g<generation>.r<rank>` (written under a temporary name, then renamed,
so a reader never sees a partial file) and reads the others' files of the
same generation.  Every rank takes the same collective steps in the same
order; a rank that does not arrive within `timeout` seconds ends the wait
with TimeoutError on the others.
"""
import os
import pickle
import time


class FileGroup:
    def __init__(self, rank, world, directory, timeout=300.0, poll=0.002):
        if world < 1 or not 0 <= rank < world:
            raise ValueError(f"rank {rank} of world {world}")
        self.rank, self.world = int(rank), int(world)
        self.dir = directory
        self.timeout = float(timeout)
        self.poll = float(poll)
        self.gen = 0
        os.makedirs(directory, exist_ok=True)

    @classmethod
    def from_env(cls, timeout=300.0):
        """The group of a job launched with RANK / WORLD_SIZE / MASTER_PORT in
        the environment (torchrun or equivalent): all ranks of one launch have
        the same parent process, which names the directory."""
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        port = os.environ.get("MASTER_PORT", "0")
        tmp = os.environ.get("TMPDIR", "/tmp")
        d = os.path.join(tmp, f"qd_group_{port}_{os.getppid()}")
        return cls(rank, world, d, timeout=timeout)

    def _path(self, gen, rank):
        return os.path.join(self.dir, f"g{gen}.r{rank}")

    def allgather(self, obj):
        """[obj of rank 0, obj of rank 1, ...] on every rank."""
        gen = self.gen
        self.gen += 1
        if self.world == 1:
            return [obj]
        mine = self._path(gen, self.rank)
        tmp = mine + ".tmp"
        with open(tmp, "wb") as f:
            pickle.dump(obj, f, protocol=pickle.HIGHEST_PROTOCOL)
        os.replace(tmp, mine)
        out = [None] * self.world
        pending = set(range(self.world))
        deadline = time.monotonic() + self.timeout
        while pending:
            for r in sorted(pending):
                p = self._path(gen, r)
                if os.path.exists(p):
                    with open(p, "rb") as f:
                        out[r] = pickle.load(f)
                    pending.discard(r)
            if pending:
                if time.monotonic() > deadline:
                    raise TimeoutError(f"rank {self.rank}: ranks {sorted(pending)} did not reach "
                                       f"collective step {gen} within {self.timeout:.0f} s")
                time.sleep(self.poll)
        # every rank has written generation gen, so every rank has finished
        # reading generation gen - 1: this rank's file of it can go
        if gen > 0:
            try:
                os.remove(self._path(gen - 1, self.rank))
            except FileNotFoundError:
                pass
        return out

    def barrier(self):
        self.allgather(None)

    def max(self, x):
        return max(self.allgather(float(x)))
