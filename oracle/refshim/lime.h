/* lime.h -- a stand-in for the c-lime calls the reference's ILDG code makes (src/io/ildg.cpp), so that
 * file compiles unchanged into the reference oracle (oracle/_ref).  TEST INFRASTRUCTURE ONLY.
 *
 * Project-written from the LIME record format (USQCD/ILDG), not c-lime.  A LIME file is a sequence
 * of records; each is a 144-byte header followed by its data, zero-padded to a multiple of 8 bytes:
 *   bytes 0-3    magic number 0x456789ab, big-endian
 *   bytes 4-5    format version 1, big-endian
 *   bytes 6-7    flags: bit 15 message begin (MB), bit 14 message end (ME), big-endian
 *   bytes 8-15   data length in bytes, big-endian
 *   bytes 16-143 record type, NUL-padded ASCII
 * Writer: a record's padding is written before the next header.  Reader: limeReaderNextRecord skips
 * the rest of the current record and its padding, reads the next header and leaves the file at the
 * start of that record's data (LIME_EOF at the end of the file or on a short or foreign header). */
#ifndef QCB_REFSHIM_LIME_H
#define QCB_REFSHIM_LIME_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t n_uint64_t;

#define LIME_SUCCESS 0
#define LIME_EOF (-1)
#define LIME_ERR_WRITE (-2)
#define LIME_ERR_READ (-3)

typedef struct {
    int mb, me;
    char type[129];
    n_uint64_t bytes;
} LimeRecordHeader;

typedef struct {
    FILE* fp;
    n_uint64_t pending_pad; /* zero bytes owed by the record being written */
} LimeWriter;

typedef struct {
    FILE* fp;
    char type[129];
    n_uint64_t bytes;
    long long data_start; /* file offset of the current record's data; -1 before the first */
} LimeReader;

static inline n_uint64_t qcb_lime_padded(n_uint64_t n) { return (n + 7u) & ~(n_uint64_t)7u; }

static inline LimeWriter* limeCreateWriter(FILE* fp) {
    LimeWriter* w = (LimeWriter*)calloc(1, sizeof(LimeWriter));
    if (w) w->fp = fp;
    return w;
}
static inline int limeDestroyWriter(LimeWriter* w) {
    free(w);
    return LIME_SUCCESS;
}
static inline LimeRecordHeader* limeCreateHeader(int MB_flag, int ME_flag, char* type, n_uint64_t reclen) {
    LimeRecordHeader* h = (LimeRecordHeader*)calloc(1, sizeof(LimeRecordHeader));
    if (!h) return h;
    h->mb = MB_flag != 0;
    h->me = ME_flag != 0;
    strncpy(h->type, type, 128);
    h->bytes = reclen;
    return h;
}
static inline void limeDestroyHeader(LimeRecordHeader* h) { free(h); }

static inline int limeWriteRecordHeader(LimeRecordHeader* h, LimeWriter* w) {
    unsigned char b[144];
    static const unsigned char zeros[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (w->pending_pad && fwrite(zeros, 1, (size_t)w->pending_pad, w->fp) != (size_t)w->pending_pad)
        return LIME_ERR_WRITE;
    w->pending_pad = 0;
    memset(b, 0, sizeof(b));
    b[0] = 0x45; b[1] = 0x67; b[2] = 0x89; b[3] = 0xab;
    b[4] = 0; b[5] = 1;
    b[6] = (unsigned char)((h->mb ? 0x80 : 0) | (h->me ? 0x40 : 0));
    b[7] = 0;
    for (int k = 0; k < 8; k++) b[8 + k] = (unsigned char)(h->bytes >> (56 - 8 * k));
    memcpy(b + 16, h->type, strlen(h->type));
    if (fwrite(b, 1, 144, w->fp) != 144) return LIME_ERR_WRITE;
    w->pending_pad = qcb_lime_padded(h->bytes) - h->bytes;
    return LIME_SUCCESS;
}
static inline int limeWriteRecordData(void* source, n_uint64_t* nbytes, LimeWriter* w) {
    return fwrite(source, 1, (size_t)*nbytes, w->fp) == (size_t)*nbytes ? LIME_SUCCESS : LIME_ERR_WRITE;
}

static inline LimeReader* limeCreateReader(FILE* fp) {
    LimeReader* r = (LimeReader*)calloc(1, sizeof(LimeReader));
    if (r) {
        r->fp = fp;
        r->data_start = -1;
    }
    return r;
}
static inline void limeDestroyReader(LimeReader* r) { free(r); }
static inline int limeReaderNextRecord(LimeReader* r) {
    unsigned char b[144];
    if (r->data_start >= 0 && fseeko(r->fp, (off_t)(r->data_start + (long long)qcb_lime_padded(r->bytes)), SEEK_SET))
        return LIME_EOF;
    if (fread(b, 1, 144, r->fp) != 144) return LIME_EOF;
    if (b[0] != 0x45 || b[1] != 0x67 || b[2] != 0x89 || b[3] != 0xab) return LIME_EOF;
    r->bytes = 0;
    for (int k = 0; k < 8; k++) r->bytes = (r->bytes << 8) | b[8 + k];
    memcpy(r->type, b + 16, 128);
    r->type[128] = 0;
    r->data_start = (long long)ftello(r->fp);
    return LIME_SUCCESS;
}
static inline char* limeReaderType(LimeReader* r) { return r->type; }
static inline n_uint64_t limeReaderBytes(LimeReader* r) { return r->bytes; }

#endif
