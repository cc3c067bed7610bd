// Loop tables of the displacement sum and the launcher interface.
//
// A plan turns the caller's loops (disco_loop) into a device table cut into
// "pieces" — a run of at most a few hundred segments (line method) or loopons
// (loopon method) of one loop, with everything that does not depend on the
// atom precomputed — packed into "chunks" that are staged whole into shared
// memory.  Pieces are independent: the field of a loop is the sum of the
// fields of its pieces (the solid angle of a convex fan splits into the solid
// angles of its sub-fans, each below 2 pi in magnitude).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/disco_b200.h"

namespace disco {

constexpr int kLineKind = 0;
constexpr int kLooponKind = 1;

// ---- FP64 line method (Code/barnett.hpp:44-107) --------------------------------
struct alignas(16) LinePiece {
    double ax, ay, az;   // vertex before the piece's first segment, minus the apex
    double cx, cy, cz;   // fan apex (loop centre)
    double bx, by, bz;   // Burgers vector (phys.b * m)
    double rho;          // largest |vertex - apex| over the piece's vertices
    double lmax;         // longest segment of the piece
    double nx, ny, nz;   // unit normal of the loop's mean plane (area vector)
    double hband;        // |n.(apex - P)| <= hband: the solid angle is taken per triangle
    int32_t nseg;        // segments of this piece
    int32_t rec;         // first segment record, index into the chunk's records
    int32_t raw;         // first of the piece's nseg + 1 input vertices in the raw array
    int32_t pad;
};
struct alignas(16) LineSeg {
    double vx, vy, vz;   // end vertex B of segment A -> B, minus the apex
    double len;          // |B - A|
    double tx, ty, tz;   // unit tangent (B - A) / |B - A| (0 for a null segment)
    double wx, wy, wz;   // w = b x t
    double nx, ny, nz;   // (A - apex) x (B - apex)
    double hl2;          // |B - A|^2 / 2
};
static_assert(sizeof(LinePiece) == 144 && sizeof(LineSeg) == 112, "line table layout");

// ---- FP64 loopon method (Code/kroupa.hpp:52-73) ---------------------------------
struct alignas(16) LooponPiece {
    double cx, cy, cz;    // reference point of the loop (loopon centroid)
    double fbx, fby, fbz; // -k1 dS b (Kroupa prefactor times the Burgers components)
    double mx, my, mz;    // unit glide direction m
    double nx, ny, nz;    // unit normal n
    double b_n;           // m . n
    int32_t n;            // loopons of this piece
    int32_t rec;          // first loopon record in the chunk
};
struct alignas(16) LooponRec {
    double x, y, z;       // loopon - reference point
    double ml, nl;        // m . (loopon - c), n . (loopon - c)
    double pad;
};
static_assert(sizeof(LooponPiece) == 112 && sizeof(LooponRec) == 48, "loopon table layout");

// ---- FP32 compensated forms -------------------------------------------------------
// Bulk arithmetic in FP32 on coordinates relative to the loop centre; the
// centre and the image offsets stay FP64.  A line piece also carries what the
// near-cut test needs (plane normal, largest vertex radius) and the index of
// the same piece in the FP64 table, which is evaluated instead for an atom
// within a few A of the loop's plane disc.
struct alignas(16) LinePieceF {
    double cx, cy, cz;       // loop centre (FP64)
    float ax, ay, az;        // start vertex - centre
    float bx, by, bz;        // Burgers vector
    float nx, ny, nz;        // unit normal of the loop plane
    float rmax;              // largest |vertex - centre| of the loop
    int32_t nseg, rec;
    int32_t piece64;         // this piece in the FP64 table
    int32_t pad;             // 80 B
};
struct alignas(16) LineSegF {
    float vx, vy, vz, len;   // end vertex - centre, length
    float tx, ty, tz;        // unit tangent
    float wx, wy, wz;        // b x t
    float nx, ny, nz;        // (start - centre) x (end - centre)
    float hl2;               // length^2 / 2
    float pad1, pad2;        // 64 B
};
static_assert(sizeof(LinePieceF) == 80 && sizeof(LineSegF) == 64, "fp32 line table layout");

struct alignas(16) LooponPieceF {
    double cx, cy, cz;      // reference point (FP64)
    float fbx, fby, fbz;    // -k1 dS b
    float mx, my, mz, nx, ny, nz;
    float b_n;
    int32_t n, rec;
    int32_t pad0, pad1;     // 80 B
};
struct alignas(16) LooponRecF {
    float x, y, z, ml;      // loopon - c, m . (loopon - c)
    float nl, pad0, pad1, pad2;   // 32 B
};
static_assert(sizeof(LooponPieceF) == 80 && sizeof(LooponRecF) == 32, "fp32 loopon table layout");

struct Chunk {
    uint64_t offset;      // byte offset of the chunk in the table
    uint32_t bytes;       // pieces then records, a multiple of 16
    int32_t npieces;
};

// Everything one launch needs; passed by value.
struct FieldArgs {
    const double *x, *y, *z;
    double *ux, *uy, *uz;
    int64_t n;
    const unsigned char* table;
    const Chunk* chunks;
    int32_t nchunks;
    uint32_t stage_bytes;     // shared-memory bytes of one stage buffer
    int32_t resident;         // one chunk, loaded once per CTA
    int32_t images, nimg;     // image range and (2 images + 1)^3
    int32_t image_min;        // skip images with max(|i|,|j|,|k|) < image_min
    int32_t pad_;
    double Lx, Ly, Lz;
    double cJ, cK;            // line: c3 - 1/(4 pi), c3 = 1 / (8 pi (1 - nu))
    double c2;                // loopon: 1 - 2 nu
    int* status;
    // FP32 line form: the FP64 pieces (flat, rec = global segment index) for
    // atoms near a loop's cut, and the near-cut distances
    const LinePiece* pieces64;
    const LineSeg* segs64;
    float near_h, near_r;
    // line method: the loops' input vertices (x, y, z triplets), read only for
    // an atom on or within hband of a loop's plane
    const double* raw;
    // FP32 line form: the atoms with at least one near-cut (piece, image).
    // near_mode 1: the FP32 pass appends them (warp-aggregated, *near_count
    // counts past near_cap); 2: the FP64 pass visits only the listed atoms, or
    // every atom when the list overflowed; 0: no list (every atom).
    int32_t* near_list;
    unsigned int* near_count;
    int32_t near_cap, near_mode;
};

// Host-side table: bytes + chunk list, built once per plan.
struct HostTable {
    int kind = kLineKind;
    bool fp32 = false;
    std::vector<unsigned char> bytes;
    std::vector<Chunk> chunks;
    uint32_t stage_bytes = 0;
    bool resident = false;
    std::vector<double> loop_evals;   // evaluations per atom per image, per input loop
    int64_t n_segments = 0, n_loopons = 0;
    // FP32 line tables: byte offsets of the flat FP64 pieces and segments
    // appended after the chunks (0 when absent)
    uint64_t aux_pieces = 0, aux_segs = 0;
    // line tables: byte offset of the raw vertex triplets (0 when absent)
    uint64_t aux_raw = 0;
};

// Appends a line table's raw vertex triplets after its chunks (sets aux_raw).
void append_raw(HostTable& T, const std::vector<double>& raw);

// Builds the table of the loops of one kind (kLineKind: loops with line != 0,
// kLooponKind: the others); returns DISCO_OK or an error code.
// stage_cap: 0 = automatic chunking, > 0 = streamed chunks of at most stage_cap
// bytes (which must hold the largest piece: 20.6 KB line, 46.2 KB loopon).
int build_table(const disco_loop* loops, int nloops, int kind, int precision, double nu,
                HostTable& out, std::string& err, uint32_t stage_cap = 0);
int build_table_fp32(const disco_loop* loops, int nloops, int kind, double nu, HostTable& out,
                     std::string& err, uint32_t stage_cap = 0);

// Picks the image split factor and grid and launches the kernel on `stream`.
int launch_field(const FieldArgs& args, int kind, bool fp32, int sm_count, int threads_hint,
                 int split_hint, cudaStream_t stream, std::string& err);

} // namespace disco
