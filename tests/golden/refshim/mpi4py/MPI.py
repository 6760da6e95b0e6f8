"""One-rank COMM_WORLD: Bcast is a no-op and Allreduce copies."""
import numpy as np

C_DOUBLE_COMPLEX = 'c16'
DOUBLE = 'f8'
INT = 'i4'
MAX = 'max'


class _Comm:
    rank = 0
    size = 1

    def Bcast(self, buf, root=0):
        return None

    def Allreduce(self, send, recv, op=None):
        np.asarray(recv[0])[...] = np.asarray(send[0])


COMM_WORLD = _Comm()
