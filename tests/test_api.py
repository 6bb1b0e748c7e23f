"""CPU tests of the drop-in Python interface (no GPU work).

Mirrors the reference's own block/texture tests (tests/test_bc1.py:15-131,
tests/test_bc4.py:14-142, tests/test_texture.py:10-60) against
quicktex_b200's classes, plus the encoder/decoder configuration surface of
s3tc/*/_bindings.cpp.
"""

import math

import pytest

import quicktex_b200 as qt
from quicktex_b200.s3tc.bc1 import BC1Block, BC1Decoder, BC1Encoder, BC1Texture
from quicktex_b200.s3tc.bc3 import BC3Block, BC3Decoder, BC3Encoder, BC3Texture
from quicktex_b200.s3tc.bc4 import BC4Block, BC4Decoder, BC4Encoder, BC4Texture
from quicktex_b200.s3tc.bc5 import BC5Block, BC5Decoder, BC5Encoder, BC5Texture
from quicktex_b200.s3tc.interpolator import Interpolator, InterpolatorAMD, InterpolatorNvidia, InterpolatorRound

BC1_BYTES = bytes.fromhex("ffff284278787878")  # tests/test_bc1.py:12
BC4_BYTES = bytes.fromhex("f010888668accffa")  # tests/test_bc4.py:9
SEL1 = [[0, 2, 3, 1]] * 4
SEL4 = [[0, 1, 2, 3]] * 2 + [[4, 5, 6, 7]] * 2


class TestBC1Block:
    def test_size(self):
        assert (BC1Block.nbytes, BC1Block.width, BC1Block.height, BC1Block.size) == (8, 4, 4, (4, 4))

    def test_buffer(self):
        b = BC1Block()
        mv = memoryview(b)
        mv[:] = BC1_BYTES
        assert not mv.readonly and mv.c_contiguous and mv.ndim == 1 and mv.nbytes == 8 and mv.format == "B"
        assert mv.tobytes() == BC1_BYTES == b.tobytes()

    def test_constructor(self):
        b = BC1Block((253, 254, 255), (65, 70, 67), SEL1)
        assert b.tobytes() == BC1_BYTES
        assert b.selectors == SEL1
        assert b.endpoints == ((255, 255, 255, 255), (66, 69, 66, 255))
        assert not b.is_3color

    def test_frombytes_eq(self):
        b = BC1Block.frombytes(BC1_BYTES)
        assert b.tobytes() == BC1_BYTES and b.selectors == SEL1
        assert b == BC1Block.frombytes(BC1_BYTES)
        assert b != BC1Block()

    def test_bad_selector(self):
        with pytest.raises(ValueError):
            BC1Block((0, 0, 0), (1, 1, 1), [[0, 1, 2, 4]] * 4)


class TestBC4Block:
    def test_size(self):
        assert (BC4Block.nbytes, BC4Block.size) == (8, (4, 4))

    def test_constructor(self):
        b = BC4Block(240, 16, SEL4)
        assert b.tobytes() == BC4_BYTES
        assert b.selectors == SEL4 and b.endpoints == (240, 16)

    def test_values(self):
        assert BC4Block(8, 248, [[0] * 4] * 4).values == [8, 248, 56, 104, 152, 200, 0, 255]
        assert BC4Block(8, 248, [[0] * 4] * 4).is_6value
        assert BC4Block(240, 16, [[0] * 4] * 4).values == [240, 16, 208, 176, 144, 112, 80, 48]
        assert not BC4Block(240, 16, [[0] * 4] * 4).is_6value

    def test_frombytes(self):
        assert BC4Block.frombytes(BC4_BYTES) == BC4Block(240, 16, SEL4)


def test_bc3_bc5_blocks():
    a, c = BC4Block.frombytes(BC4_BYTES), BC1Block.frombytes(BC1_BYTES)
    b3 = BC3Block(a, c)
    assert b3.tobytes() == BC4_BYTES + BC1_BYTES and BC3Block.nbytes == 16
    assert b3.alpha_block == a and b3.color_block == c and b3.blocks == (a, c)
    b5 = BC5Block(a, BC4Block())
    assert b5.tobytes() == BC4_BYTES + bytes(8) and b5.chan0_block == a
    b5.blocks = (BC4Block(), a)
    assert b5.tobytes() == bytes(8) + BC4_BYTES


@pytest.mark.parametrize("tex_cls,blk_cls", [(BC1Texture, BC1Block), (BC4Texture, BC4Block), (BC3Texture, BC3Block),
                                             (BC5Texture, BC5Block)])
@pytest.mark.parametrize("w", [7, 8, 9])
@pytest.mark.parametrize("h", [7, 8, 9])
class TestBlockTexture:
    def test_dimensions(self, tex_cls, blk_cls, w, h):
        tex = tex_cls(w, h)
        wb, hb = math.ceil(w / 4), math.ceil(h / 4)
        assert tex.nbytes == blk_cls.nbytes * wb * hb == len(tex.tobytes())
        assert (tex.width, tex.height, tex.size) == (w, h, (w, h))
        assert (tex.width_blocks, tex.height_blocks, tex.size_blocks) == (wb, hb, (wb, hb))

    def test_blocks(self, tex_cls, blk_cls, w, h):
        tex = tex_cls(w, h)
        n = blk_cls.nbytes
        blocks = [[blk_cls.frombytes(bytes([x, y] + [0] * (n - 2))) for x in range(tex.width_blocks)]
                  for y in range(tex.height_blocks)]
        for x in range(tex.width_blocks):
            for y in range(tex.height_blocks):
                tex[x, y] = blocks[y][x]
        raw = tex.tobytes()
        for x in range(tex.width_blocks):
            for y in range(tex.height_blocks):
                i = (x + y * tex.width_blocks) * n
                assert tex[x, y] == blocks[y][x] == blk_cls.frombytes(raw[i:i + n])

    def test_subscript(self, tex_cls, blk_cls, w, h):
        tex = tex_cls(w, h)
        assert tex[-1, -1] == tex[tex.width_blocks - 1, tex.height_blocks - 1]
        with pytest.raises(IndexError):
            _ = tex[tex.width_blocks, tex.height_blocks]
        with pytest.raises(IndexError):
            _ = tex[-1 - tex.width_blocks, -1 - tex.height_blocks]

    def test_buffer(self, tex_cls, blk_cls, w, h):
        tex = tex_cls(w, h)
        mv = memoryview(tex)
        data = bytes(range(256)) * (tex.nbytes // 256 + 1)
        data = data[:tex.nbytes]
        mv[:] = data
        assert not mv.readonly and mv.c_contiguous and mv.nbytes == tex.nbytes and mv.format == "B"
        assert mv.tobytes() == data
        assert tex_cls.from_bytes(data, w, h).tobytes() == data


class TestRawTexture:
    W, H = 37, 19

    def test_size(self):
        t = qt.RawTexture(self.W, self.H)
        assert t.nbytes == self.W * self.H * 4 and t.size == (self.W, self.H)

    def test_pixels(self):
        t = qt.RawTexture(self.W, self.H)
        c1, c2 = (69, 13, 12, 0), (19, 142, 93, 44)
        t[0, 0] = c1
        t[-1, -1] = c2
        d = t.tobytes()
        assert t[0, 0] == c1 and t[-1, -1] == c2
        assert tuple(d[0:4]) == c1 and tuple(d[-4:]) == c2
        t[1, 0] = (1, 2, 3)
        assert t[1, 0] == (1, 2, 3, 255)
        with pytest.raises(IndexError):
            _ = t[self.W, self.H]
        with pytest.raises(IndexError):
            _ = t[-1 - self.W, -1 - self.H]
        with pytest.raises(TypeError):
            t[0, 0] = (1, 2, 300)

    def test_buffer_frombytes(self):
        data = bytes((i * 7) & 255 for i in range(self.W * self.H * 4))
        t = qt.RawTexture(self.W, self.H)
        memoryview(t)[:] = data
        assert t.tobytes() == data
        assert qt.RawTexture.frombytes(data, self.W, self.H).tobytes() == data
        with pytest.raises(RuntimeError):
            qt.RawTexture.frombytes(data[:-1], self.W, self.H)

    def test_bad_dims(self):
        with pytest.raises(ValueError):
            qt.RawTexture(0, 4)
        with pytest.raises(ValueError):
            BC1Texture(4, -1)


class TestEncoderSurface:
    def test_bc1_defaults(self):
        e = BC1Encoder()
        assert e.color_mode == BC1Encoder.ColorMode.FourColor
        assert isinstance(e.interpolator, Interpolator)
        # level 5 (BC1Encoder.cpp:114-118): two LS passes, Faster, PCA, one ordering each
        assert e.error_mode == BC1Encoder.ErrorMode.Faster and e.endpoint_mode == BC1Encoder.EndpointMode.PCA
        assert e.two_ls_passes and not e.two_ep_passes and not e.two_cf_passes and not e.exhaustive
        assert e.orderings == (1, 1) and e.search_rounds == 0 and e.power_iterations == 4

    def test_bc1_levels_and_setters(self):
        e = BC1Encoder(18, BC1Encoder.ColorMode.ThreeColorBlack, InterpolatorAMD())
        assert e.orderings == (128, 32) and e.search_rounds == 256 and e.two_cf_passes
        assert isinstance(e.interpolator, InterpolatorAMD)
        e.set_level(0)
        assert e.endpoint_mode == BC1Encoder.EndpointMode.BoundingBoxInt and e.orderings == (1, 1)
        e.orderings = (500, 0)
        assert e.orderings == (128, 1)
        e.power_iterations = 99
        assert e.power_iterations == BC1Encoder.max_power_iterations == 10
        e.power_iterations = 0
        assert e.power_iterations == BC1Encoder.min_power_iterations == 4
        e.error_mode = getattr(BC1Encoder.ErrorMode, "None")
        assert int(e.error_mode) == 0
        with pytest.raises(ValueError):
            e.set_level(20)
        e.set_level(19)  # the hidden exhaustive level is accepted
        assert e.exhaustive

    def test_interpolator_classes(self):
        for cls in (Interpolator, InterpolatorRound, InterpolatorNvidia, InterpolatorAMD):
            assert isinstance(cls(), Interpolator)

    def test_other_codecs(self):
        assert BC4Encoder().channel == 3 and BC4Encoder(1).channel == 1 and BC4Decoder(2).channel == 2
        with pytest.raises(ValueError):
            BC4Encoder(4)
        with pytest.raises(ValueError):
            BC4Decoder(7)
        b5 = BC5Encoder(2, 0)
        assert b5.channels == (2, 0) and [x.channel for x in b5.bc4_encoders] == [2, 0]
        assert BC5Decoder().channels == (0, 1)
        b3 = BC3Encoder(10, InterpolatorRound())
        assert b3.bc1_encoder.color_mode == BC1Encoder.ColorMode.FourColor and b3.bc4_encoder.channel == 3
        assert isinstance(b3.bc1_encoder.interpolator, InterpolatorRound) and b3.bc1_encoder.orderings == (20, 8)
        d3 = BC3Decoder(InterpolatorNvidia())
        assert isinstance(d3.bc1_decoder.interpolator, InterpolatorNvidia) and d3.bc4_decoder.channel == 3
        d1 = BC1Decoder()
        assert not d1.write_alpha
        d1.write_alpha = True
        assert d1.write_alpha and BC1Decoder(True, InterpolatorAMD()).write_alpha
