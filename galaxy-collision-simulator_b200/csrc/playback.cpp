// playback.cpp - reading simulation.bin back frame by frame: the reference's
// Playback mode (main.cpp:299-453) without its window.
//
// A simulation.bin file is a sequence of frames of PlaybackStar records
// (16 bytes: x, y, z, r, g, b, type), one record per particle, as the Bake
// loop writes them (main.cpp:264-272) and gcs_bake / the server write them
// here.  The reference recovers the particle count by assuming 2000 frames
// (main.cpp:309); a reader opened with the particle count instead derives the
// frame count from the file size and rejects a size that is not a whole
// number of frames.  The reference's inference stays available (particles
// = 0 with its frame count as the hint).
//
// Navigation follows the reference's file-offset arithmetic, with the file
// offset kept in frames, o in [0, frames] (frames: at the end of the file):
//   * forward (main.cpp:413-419): read frame o and move to o + 1; at the end
//     of the file the read loops to frame 0;
//   * backward (main.cpp:397-410): move back two frames, to o - 2, or to the
//     last frame when that is negative; then read that frame (the reference
//     moves to the file size minus one frame, which is the last whole frame
//     when the size is a whole number of frames);
//   * the per-frame camera target is the FP64 mean position, rounded to
//     float (main.cpp:435-441).
#include <cstdint>
#include <cstdio>
#include <new>

#include "../../include/gcs.h"

struct gcs_playback {
    FILE* file = nullptr;
    int64_t particles = 0;
    int64_t frames = 0;
    int64_t offset = 0;  // file offset in frames, 0 .. frames (the end)
};

namespace {

int read_frame(gcs_playback* pb, int64_t frame, PlaybackStar* host) {
    const int64_t bytes = pb->particles * (int64_t)sizeof(PlaybackStar);
    if (fseeko(pb->file, (off_t)(frame * bytes), SEEK_SET) != 0) return GCS_ERR_ARG;
    if (fread(host, sizeof(PlaybackStar), (size_t)pb->particles, pb->file) != (size_t)pb->particles)
        return GCS_ERR_ARG;
    return GCS_OK;
}

}  // namespace

extern "C" {

int gcs_playback_open(const char* path, int64_t particles, int64_t frames_hint, gcs_playback** out) {
    if (!path || !out || particles < 0 || (particles == 0 && frames_hint < 1)) return GCS_ERR_ARG;
    *out = nullptr;
    FILE* f = std::fopen(path, "rb");
    if (!f) return GCS_ERR_ARG;
    int64_t size = -1;
    if (fseeko(f, 0, SEEK_END) == 0) size = (int64_t)ftello(f);
    if (size <= 0) {
        std::fclose(f);
        return GCS_ERR_ARG;
    }
    const int64_t rec = (int64_t)sizeof(PlaybackStar);
    int64_t n = particles;
    if (n == 0) {
        n = size / frames_hint / rec;  // main.cpp:309 with the hint for its 2000
    } else if (size % (n * rec) != 0) {
        std::fclose(f);  // not a whole number of frames of n particles
        return GCS_ERR_ARG;
    }
    if (n <= 0 || size / (n * rec) < 1) {
        std::fclose(f);
        return GCS_ERR_ARG;
    }
    gcs_playback* pb = new (std::nothrow) gcs_playback;
    if (!pb) {
        std::fclose(f);
        return GCS_ERR_NOMEM;
    }
    pb->file = f;
    pb->particles = n;
    pb->frames = size / (n * rec);  // whole frames (the inference may leave a remainder)
    pb->offset = 0;
    *out = pb;
    return GCS_OK;
}

int64_t gcs_playback_frames(const gcs_playback* pb) { return pb ? pb->frames : 0; }
int64_t gcs_playback_particles(const gcs_playback* pb) { return pb ? pb->particles : 0; }
int64_t gcs_playback_position(const gcs_playback* pb) { return pb ? pb->offset % pb->frames : 0; }

int gcs_playback_seek(gcs_playback* pb, int64_t frame) {
    if (!pb) return GCS_ERR_ARG;
    const int64_t m = frame % pb->frames;
    pb->offset = m < 0 ? m + pb->frames : m;
    return GCS_OK;
}

int gcs_playback_next(gcs_playback* pb, PlaybackStar* host) {
    if (!pb || !host) return GCS_ERR_ARG;
    const int64_t f = pb->offset == pb->frames ? 0 : pb->offset;  // loop at the end of the file
    const int rc = read_frame(pb, f, host);
    if (rc) return rc;
    pb->offset = f + 1;
    return GCS_OK;
}

int gcs_playback_prev(gcs_playback* pb, PlaybackStar* host) {
    if (!pb || !host) return GCS_ERR_ARG;
    int64_t f = pb->offset - 2;
    if (f < 0) f = pb->frames - 1;
    const int rc = read_frame(pb, f, host);
    if (rc) return rc;
    pb->offset = f + 1;
    return GCS_OK;
}

int gcs_playback_centre(const PlaybackStar* frame, int64_t n, float centre[3]) {
    if (!frame || n <= 0 || !centre) return GCS_ERR_ARG;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        sx += frame[i].x;
        sy += frame[i].y;
        sz += frame[i].z;
    }
    centre[0] = (float)(sx / (double)n);
    centre[1] = (float)(sy / (double)n);
    centre[2] = (float)(sz / (double)n);
    return GCS_OK;
}

void gcs_playback_close(gcs_playback* pb) {
    if (!pb) return;
    if (pb->file) std::fclose(pb->file);
    delete pb;
}

}  // extern "C"
