// strip_tiles.h — how the learned absorbing strip is cut into tiles (host
// code; learned.cu builds the tile list with it, and a CPU test compiles it
// on its own to check the cover and the staging bounds).
#pragma once

#include <algorithm>
#include <vector>

#include <vector_functions.h>   // make_int4

namespace sgfd {

constexpr int kStripRows = 128;    // cells per tile: the tensor-core tile's M
constexpr int kStripStage = 544;   // staged cells of a box with its one-cell halo, at most: (32+2)(2+2)(2+2)

// Boxes of at most kStripRows strip cells covering the strip of width w of an
// X x Y x Z computed region exactly once: the two z faces and the two y faces
// (between the z faces) in 32 x 2 x 2 boxes, the two x faces (between the
// others) in min(w, 32) x ey x ez (6 x 4 x 5 for w = 6).  Each tile is
// (x, y, z, ex | ey << 8 | ez << 16) in computed coordinates, the extents
// clipped at the faces' ends.  Returns the number of tiles, or -1 if a box
// with its halo would not fit kStripStage.  Needs 1 <= w and 2w < X, Y, Z.
inline int strip_tiles(int X, int Y, int Z, int w, std::vector<int4> &tiles) {
    tiles.clear();
    bool fits = true;
    auto boxes = [&](int x0, int x1, int y0, int y1, int z0, int z1, int ex, int ey, int ez) {
        fits = fits && ex * ey * ez <= kStripRows && (ex + 2) * (ey + 2) * (ez + 2) <= kStripStage;
        for (int z = z0; z < z1; z += ez)
            for (int y = y0; y < y1; y += ey)
                for (int x = x0; x < x1; x += ex)
                    tiles.push_back(make_int4(x, y, z, std::min(ex, x1 - x) | std::min(ey, y1 - y) << 8 |
                                                           std::min(ez, z1 - z) << 16));
    };
    boxes(0, X, 0, Y, 0, w, 32, 2, 2);
    boxes(0, X, 0, Y, Z - w, Z, 32, 2, 2);
    boxes(0, X, 0, w, w, Z - w, 32, 2, 2);
    boxes(0, X, Y - w, Y, w, Z - w, 32, 2, 2);
    const int ex = std::min(w, 32), rest = kStripRows / ex;
    int ey = 1;
    while (4 * ey * ey <= rest) ey *= 2;   // largest power of two with ey^2 <= rest
    const int ez = rest / ey;
    boxes(0, w, w, Y - w, w, Z - w, ex, ey, ez);
    boxes(X - w, X, w, Y - w, w, Z - w, ex, ey, ez);
    return fits ? (int)tiles.size() : -1;
}

}  // namespace sgfd
