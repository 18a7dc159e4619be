"""Public types of the crate: CompressionVariant and the BC6H/BC7 quality
profiles (src/lib.rs:67-198, src/settings.rs:199-442), as ctypes structures
with the reference's #[repr(C)] byte layout so they cross the C ABI as-is."""
import ctypes

from ._lib import check, lib


class BC6HSettings(ctypes.Structure):
    """Encoding settings for BC6H (src/settings.rs:207-213)."""

    _fields_ = [
        ("slow_mode", ctypes.c_uint32),
        ("fast_mode", ctypes.c_uint32),
        ("refine_iterations_1p", ctypes.c_uint32),
        ("refine_iterations_2p", ctypes.c_uint32),
        ("fast_skip_threshold", ctypes.c_uint32),
    ]

    @classmethod
    def _preset(cls, name):
        s = cls()
        check("bc_bc6h_settings_preset", lib.bc_bc6h_settings_preset(name.encode(), ctypes.byref(s)))
        return s

    @classmethod
    def very_fast(cls):
        return cls._preset("very_fast")

    @classmethod
    def fast(cls):
        return cls._preset("fast")

    @classmethod
    def basic(cls):
        return cls._preset("basic")

    @classmethod
    def slow(cls):
        return cls._preset("slow")

    @classmethod
    def very_slow(cls):
        return cls._preset("very_slow")

    def as_list(self):
        return [self.slow_mode, self.fast_mode, self.refine_iterations_1p, self.refine_iterations_2p,
                self.fast_skip_threshold]

    def __eq__(self, other):
        return isinstance(other, BC6HSettings) and self.as_list() == other.as_list()

    def __repr__(self):
        return "BC6HSettings(%s)" % ", ".join("%s=%d" % (n, getattr(self, n)) for n, _ in self._fields_)


class BC7Settings(ctypes.Structure):
    """Encoding settings for BC7 (src/settings.rs:278-288)."""

    _fields_ = [
        ("refine_iterations", ctypes.c_uint32 * 8),
        ("mode_selection", ctypes.c_uint32 * 4),
        ("skip_mode2", ctypes.c_uint32),
        ("fast_skip_threshold_mode1", ctypes.c_uint32),
        ("fast_skip_threshold_mode3", ctypes.c_uint32),
        ("fast_skip_threshold_mode7", ctypes.c_uint32),
        ("mode45_channel0", ctypes.c_uint32),
        ("refine_iterations_channel", ctypes.c_uint32),
        ("channels", ctypes.c_uint32),
    ]

    @classmethod
    def _preset(cls, name):
        s = cls()
        check("bc_bc7_settings_preset", lib.bc_bc7_settings_preset(name.encode(), ctypes.byref(s)))
        return s

    @classmethod
    def opaque_ultra_fast(cls):
        return cls._preset("opaque_ultra_fast")

    @classmethod
    def opaque_very_fast(cls):
        return cls._preset("opaque_very_fast")

    @classmethod
    def opaque_fast(cls):
        return cls._preset("opaque_fast")

    @classmethod
    def opaque_basic(cls):
        return cls._preset("opaque_basic")

    @classmethod
    def opaque_slow(cls):
        return cls._preset("opaque_slow")

    @classmethod
    def alpha_ultrafast(cls):
        return cls._preset("alpha_ultrafast")

    @classmethod
    def alpha_very_fast(cls):
        return cls._preset("alpha_very_fast")

    @classmethod
    def alpha_fast(cls):
        return cls._preset("alpha_fast")

    @classmethod
    def alpha_basic(cls):
        return cls._preset("alpha_basic")

    @classmethod
    def alpha_slow(cls):
        return cls._preset("alpha_slow")

    def as_list(self):
        return (list(self.refine_iterations) + list(self.mode_selection) +
                [self.skip_mode2, self.fast_skip_threshold_mode1, self.fast_skip_threshold_mode3,
                 self.fast_skip_threshold_mode7, self.mode45_channel0, self.refine_iterations_channel,
                 self.channels])

    def __eq__(self, other):
        return isinstance(other, BC7Settings) and self.as_list() == other.as_list()

    def __repr__(self):
        return "BC7Settings(%s)" % self.as_list()


class CompressionVariant:
    """Block compression variant (src/lib.rs:74-103).

    BC1..BC5 are singletons; BC6H and BC7 carry settings. Like the reference,
    equality and hashing look at the variant kind only (src/lib.rs:106-120).
    """

    _NAMES = ("BC1", "BC2", "BC3", "BC4", "BC5", "BC6H", "BC7")
    __slots__ = ("id", "settings")

    def __init__(self, vid, settings=None):
        self.id = vid
        self.settings = settings

    @classmethod
    def BC6H(cls, settings):
        return cls(5, settings)

    @classmethod
    def BC7(cls, settings):
        return cls(6, settings)

    @property
    def name(self):
        return self._NAMES[self.id]

    def block_byte_size(self):
        return 8 if self.id in (0, 3) else 16

    def bytes_per_row(self, width):
        """src/lib.rs:129-132"""
        return lib.bc_bytes_per_row(self.id, width)

    def blocks_byte_size(self, width, height):
        """src/lib.rs:138-144"""
        return lib.bc_blocks_byte_size(self.id, width, height)

    def settings_ptr(self):
        return ctypes.cast(ctypes.byref(self.settings), ctypes.c_void_p) if self.settings is not None else None

    def __eq__(self, other):
        return isinstance(other, CompressionVariant) and other.id == self.id

    def __hash__(self):
        return hash(self.id)

    def __repr__(self):
        return self.name if self.settings is None else "%s(%r)" % (self.name, self.settings)


CompressionVariant.BC1 = CompressionVariant(0)
CompressionVariant.BC2 = CompressionVariant(1)
CompressionVariant.BC3 = CompressionVariant(2)
CompressionVariant.BC4 = CompressionVariant(3)
CompressionVariant.BC5 = CompressionVariant(4)
