"""Single-rank MPI communicator: every collective is the identity."""
import numpy as _np

SUM = "sum"
MAX = "max"
MIN = "min"
IN_PLACE = object()
DOUBLE = "double"
INT = "int"


class _Comm:
    rank = 0
    size = 1

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def barrier(self):
        return None

    Barrier = barrier

    def allgather(self, x):
        return [x]

    def gather(self, x, root=0):
        return [x]

    def bcast(self, x, root=0):
        return x

    def reduce(self, x, op=SUM, root=0):
        return x

    def allreduce(self, x, op=SUM):
        return x

    def Allreduce(self, sendbuf, recvbuf=None, op=SUM):
        if sendbuf is IN_PLACE:
            return None
        _np.copyto(_np.asarray(recvbuf), _np.asarray(sendbuf).reshape(_np.shape(recvbuf)))

    def Allgather(self, sendbuf, recvbuf):
        _np.asarray(recvbuf)[...] = _np.asarray(sendbuf).reshape(_np.shape(recvbuf))

    def Allgatherv(self, sendbuf, recvbuf):
        buf = recvbuf[0] if isinstance(recvbuf, (list, tuple)) else recvbuf
        src = sendbuf[0] if isinstance(sendbuf, (list, tuple)) else sendbuf
        _np.asarray(buf).reshape(-1)[: _np.size(src)] = _np.asarray(src).reshape(-1)

    def Abort(self, code=1):
        raise SystemExit(code)


COMM_WORLD = _Comm()
