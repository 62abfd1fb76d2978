"""Error type of the native calls, drop-in for tigre.utilities.errors (errors.py:8-25)."""


class Error(Exception):
    pass


class TigreCudaCallError(Error):
    """Indexed against the codes of Common/CUDA/errors.hpp (1..5)."""

    _messages = [
        "GPU: Cuda error with exit code 1.",
        "There are no available device(s) that support CUDA",
        "GPU: One (or more) of your GPUs is being heavily used by another program (possibly graphics-based).\n"
        "Free the GPU to run TIGRE",
        "GPU: Assertion Failed. Logic behind splitting flawed! Please tell: ander.biguri@gmail.com",
        "GPU: Assertion Failed. Memory needed calculation broken! Please tell: ander.biguri@gmail.com",
    ]

    def __init__(self, txt, error_index, detail=""):
        Error.__init__(self)
        self.txt = txt
        self.error_index = error_index
        self.detail = detail

    def __str__(self):
        i = self.error_index - 1
        msg = self._messages[i] if 0 <= i < len(self._messages) else "unknown error %d" % self.error_index
        return "\n".join([self.txt, msg] + ([self.detail] if self.detail else []))
