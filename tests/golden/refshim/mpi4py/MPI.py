"""One-rank ``mpi4py.MPI``: the calls the reference makes at one rank
(topology.py Create_cart/Shift, solver.py allreduce, run.py Barrier)."""

MAX = "max"
MIN = "min"
PROC_NULL = -2


class _Cart:
    def Shift(self, axis, disp):
        return (PROC_NULL, PROC_NULL)


class Comm:
    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def Create_cart(self, dims, periods=None, reorder=False):
        return _Cart()

    def allreduce(self, x, op=None):
        return x

    def Barrier(self):
        return None


COMM_WORLD = Comm()
