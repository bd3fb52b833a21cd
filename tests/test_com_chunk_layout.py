"""The row-end rule the COM-only kernel's u16 fast path relies on (com.cu:chunk_moments_u16): its
16-byte chunks hold 8 pixels and start at pixel 8c of the ROI, so a chunk starts at column
x0 = 8c mod W. With W a multiple of 8 no chunk crosses a row end; with W = 8k + 4 a chunk that
crosses one does so after its fourth pixel (split W - x0 = 4), so the pixels on the next row are the
chunk's second half. Checked by enumeration over the widths the kernel accepts (W >= 8)."""


def crossing_splits(W: int, H: int) -> set:
    splits = set()
    for c in range(W * H // 8):
        x0 = (8 * c) % W
        if x0 + 8 > W:
            splits.add(W - x0)
    return splits


def test_rows_of_a_multiple_of_8_pixels_are_never_crossed():
    for W in range(8, 520, 8):
        assert crossing_splits(W, 8) == set(), W


def test_rows_of_8k_plus_4_pixels_are_crossed_after_the_fourth_pixel():
    for W in range(12, 524, 8):
        assert crossing_splits(W, 8) == {4}, W


def test_other_widths_need_the_general_split():
    for W in (9, 10, 50, 99, 101, 130):
        assert crossing_splits(W, 16) - {4}, W
