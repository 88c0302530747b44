"""Single-rank MPI stand-in: COMM_WORLD has rank 0 of size 1, datatypes are
opaque tokens.  Only what lcode/mpi/{transport,util}.py touch at import time
and on the single-process path is provided; any send/recv raises."""


class Datatype:
    def __init__(self, name="struct"):
        self.name = name

    @staticmethod
    def Create_struct(*args, **kwargs):
        return Datatype()

    def Create_resized(self, *args, **kwargs):
        return self

    def Commit(self):
        return self


for _n in ("INT8_T", "INT16_T", "INT32_T", "INT64_T", "UINT8_T", "UINT16_T",
           "UINT32_T", "UINT64_T", "FLOAT", "DOUBLE"):
    globals()[_n] = Datatype(_n)


class Status:
    def Get_count(self, datatype=None):
        raise RuntimeError("single-rank MPI stand-in has no messages")


class _Comm:
    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def Send(self, *a, **k):
        raise RuntimeError("single-rank MPI stand-in cannot send")

    def Recv(self, *a, **k):
        raise RuntimeError("single-rank MPI stand-in cannot receive")

    def Probe(self, *a, **k):
        raise RuntimeError("single-rank MPI stand-in cannot probe")


COMM_WORLD = _Comm()
Comm = _Comm
