/*
 * The on-disk container of the checkpoint: a NumPy .npz archive (an
 * uncompressed ZIP whose members are .npy arrays), written and read here in
 * plain C so that the C ABI can write and restart from checkpoints without
 * Python.  Member names are the reference's HDF5 dataset paths
 * ("Grid/T.npy", "Data/Cells.npy", ... of Output/h5out.c), so
 * numpy.load(path)["Data/Cells"] reads what h5py's f["Data"]["Cells"] would.
 *
 * ZIP (PKWARE APPNOTE 6.3): every member is stored (method 0) and carries
 * ZIP64 extra fields, so members and archives larger than 4 GiB need no
 * special case; the archive ends with a ZIP64 end-of-central-directory record
 * and locator.  The member CRC-32 is zlib's.  .npy (NEP 1 format, version
 * 1.0): magic, header length, a Python-literal dict with descr /
 * fortran_order / shape, padded with spaces to a multiple of 64 bytes.
 */
#include "disco_host.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

#define NPZ_MAXMEM 4096

struct npz_member {
   char *name;
   uint64_t offset;          /* of the local header */
   uint64_t size;            /* stored bytes (npy header + data) */
   uint32_t crc;
   uint64_t data_off;        /* of the array data (reader, lazily) */
   uint64_t data_bytes;      /* array data bytes (reader, lazily) */
};

struct disco_npz {
   FILE *f;
   int writing;
   int nmem;
   struct npz_member mem[NPZ_MAXMEM];
   /* the member being written */
   int open;
   uint64_t expect, written;
   uint32_t crc;
};

static void put16(unsigned char *p, unsigned v){ p[0] = v & 255; p[1] = (v >> 8) & 255; }
static void put32(unsigned char *p, uint32_t v){ for( int i=0 ; i<4 ; ++i ) p[i] = (v >> (8*i)) & 255; }
static void put64(unsigned char *p, uint64_t v){ for( int i=0 ; i<8 ; ++i ) p[i] = (v >> (8*i)) & 255; }
static unsigned get16(const unsigned char *p){ return p[0] | (p[1] << 8); }
static uint32_t get32(const unsigned char *p){
   return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static uint64_t get64(const unsigned char *p){ return (uint64_t)get32(p) | ((uint64_t)get32(p+4) << 32); }

static int itemsize(const char *descr){
   if( !descr || strlen(descr) < 3 ) return 0;
   if( descr[0] != '<' && descr[0] != '|' && descr[0] != '=' ) return 0;
   return atoi(descr + 2);
}

/* the .npy v1.0 header for an array of this descr and shape; returns its
 * length (a multiple of 64) */
static size_t npy_header(char *out, size_t cap, const char *descr, int ndim, const int64_t *shape){
   char dict[512], sh[256] = "(";
   int n = 1;
   for( int d=0 ; d<ndim ; ++d )
      n += snprintf(sh + n, sizeof sh - n, d ? ", %lld" : "%lld", (long long)shape[d]);
   snprintf(sh + n, sizeof sh - n, ndim == 1 ? ",)" : ")");
   int len = snprintf(dict, sizeof dict, "{'descr': '%s', 'fortran_order': False, 'shape': %s, }",
                      descr, sh);
   size_t total = 10 + (size_t)len + 1;
   total = (total + 63) / 64 * 64;
   if( total > cap ) return 0;
   memcpy(out, "\x93NUMPY\x01\x00", 8);
   put16((unsigned char *)out + 8, (unsigned)(total - 10));
   memcpy(out + 10, dict, len);
   memset(out + 10 + len, ' ', total - 10 - len - 1);
   out[total - 1] = '\n';
   return total;
}

int disco_npz_create(const char *path, disco_npz **out){
   if( !path || !out ) return DISCO_ERR_ARG;
   *out = NULL;
   disco_npz *z = (disco_npz *)calloc(1, sizeof *z);
   if( !z ) return DISCO_ERR_IO;
   z->f = fopen(path, "wb");
   if( !z->f ){ free(z); return DISCO_ERR_IO; }
   z->writing = 1;
   *out = z;
   return DISCO_OK;
}

int disco_npz_begin(disco_npz *z, const char *name, const char *descr, int ndim, const int64_t *shape){
   if( !z || !z->writing || z->open || !name || !descr || ndim < 0 || ndim > 8 ) return DISCO_ERR_ARG;
   if( z->nmem >= NPZ_MAXMEM ) return DISCO_ERR_ARG;
   int isz = itemsize(descr);
   if( isz <= 0 ) return DISCO_ERR_ARG;
   uint64_t count = 1;
   for( int d=0 ; d<ndim ; ++d ){ if( shape[d] < 0 ) return DISCO_ERR_ARG; count *= (uint64_t)shape[d]; }
   char hdr[1024];
   size_t hl = npy_header(hdr, sizeof hdr, descr, ndim, shape);
   if( !hl ) return DISCO_ERR_ARG;
   char fname[600];
   int nl = snprintf(fname, sizeof fname, "%s.npy", name);
   if( nl <= 0 || nl >= (int)sizeof fname ) return DISCO_ERR_ARG;
   struct npz_member *m = &z->mem[z->nmem];
   m->name = strdup(fname);
   if( !m->name ) return DISCO_ERR_IO;
   m->offset = (uint64_t)ftello(z->f);
   m->size = hl + count*(uint64_t)isz;
   /* local file header + ZIP64 extra (sizes); CRC patched in disco_npz_end */
   unsigned char lh[30 + 20];
   put32(lh, 0x04034b50u); put16(lh + 4, 45); put16(lh + 6, 0); put16(lh + 8, 0);
   put16(lh + 10, 0); put16(lh + 12, 0x21);
   put32(lh + 14, 0); put32(lh + 18, 0xffffffffu); put32(lh + 22, 0xffffffffu);
   put16(lh + 26, (unsigned)nl); put16(lh + 28, 20);
   unsigned char *ex = lh + 30;
   put16(ex, 1); put16(ex + 2, 16); put64(ex + 4, m->size); put64(ex + 12, m->size);
   if( fwrite(lh, 1, 30, z->f) != 30 || fwrite(fname, 1, nl, z->f) != (size_t)nl ||
       fwrite(ex, 1, 20, z->f) != 20 ) return DISCO_ERR_IO;
   z->open = 1;
   z->expect = m->size;
   z->written = 0;
   z->crc = (uint32_t)crc32_z(0L, Z_NULL, 0);
   return disco_npz_append(z, hdr, hl);
}

int disco_npz_append(disco_npz *z, const void *data, size_t nbytes){
   if( !z || !z->open ) return DISCO_ERR_ARG;
   if( nbytes == 0 ) return DISCO_OK;
   if( !data || z->written + nbytes > z->expect ) return DISCO_ERR_ARG;
   z->crc = (uint32_t)crc32_z(z->crc, (const Bytef *)data, nbytes);
   if( fwrite(data, 1, nbytes, z->f) != nbytes ) return DISCO_ERR_IO;
   z->written += nbytes;
   return DISCO_OK;
}

int disco_npz_end(disco_npz *z){
   if( !z || !z->open ) return DISCO_ERR_ARG;
   z->open = 0;
   struct npz_member *m = &z->mem[z->nmem];
   if( z->written != z->expect ) return DISCO_ERR_ARG;
   m->crc = z->crc;
   unsigned char b[4];
   put32(b, m->crc);
   off_t end = ftello(z->f);
   if( fseeko(z->f, (off_t)m->offset + 14, SEEK_SET) || fwrite(b, 1, 4, z->f) != 4 ||
       fseeko(z->f, end, SEEK_SET) ) return DISCO_ERR_IO;
   z->nmem++;
   return DISCO_OK;
}

int disco_npz_put(disco_npz *z, const char *name, const char *descr, int ndim,
                  const int64_t *shape, const void *data){
   int s = disco_npz_begin(z, name, descr, ndim, shape);
   if( s ) return s;
   size_t hl = (size_t)z->written;
   s = disco_npz_append(z, data, (size_t)(z->expect - hl));
   if( s ) return s;
   return disco_npz_end(z);
}

static int write_directory(disco_npz *z){
   uint64_t cd_off = (uint64_t)ftello(z->f);
   for( int i=0 ; i<z->nmem ; ++i ){
      struct npz_member *m = &z->mem[i];
      size_t nl = strlen(m->name);
      unsigned char c[46 + 28];
      put32(c, 0x02014b50u); put16(c + 4, 45); put16(c + 6, 45); put16(c + 8, 0);
      put16(c + 10, 0); put16(c + 12, 0); put16(c + 14, 0x21);
      put32(c + 16, m->crc); put32(c + 20, 0xffffffffu); put32(c + 24, 0xffffffffu);
      put16(c + 28, (unsigned)nl); put16(c + 30, 28); put16(c + 32, 0);
      put16(c + 34, 0); put16(c + 36, 0); put32(c + 38, 0); put32(c + 42, 0xffffffffu);
      unsigned char *ex = c + 46;
      put16(ex, 1); put16(ex + 2, 24);
      put64(ex + 4, m->size); put64(ex + 12, m->size); put64(ex + 20, m->offset);
      if( fwrite(c, 1, 46, z->f) != 46 || fwrite(m->name, 1, nl, z->f) != nl ||
          fwrite(ex, 1, 28, z->f) != 28 ) return DISCO_ERR_IO;
   }
   uint64_t cd_end = (uint64_t)ftello(z->f);
   unsigned char e64[56], loc[20], eocd[22];
   put32(e64, 0x06064b50u); put64(e64 + 4, 44); put16(e64 + 12, 45); put16(e64 + 14, 45);
   put32(e64 + 16, 0); put32(e64 + 20, 0);
   put64(e64 + 24, (uint64_t)z->nmem); put64(e64 + 32, (uint64_t)z->nmem);
   put64(e64 + 40, cd_end - cd_off); put64(e64 + 48, cd_off);
   put32(loc, 0x07064b50u); put32(loc + 4, 0); put64(loc + 8, cd_end); put32(loc + 16, 1);
   put32(eocd, 0x06054b50u); put16(eocd + 4, 0); put16(eocd + 6, 0);
   put16(eocd + 8, 0xffff); put16(eocd + 10, 0xffff);
   put32(eocd + 12, 0xffffffffu); put32(eocd + 16, 0xffffffffu); put16(eocd + 20, 0);
   if( fwrite(e64, 1, 56, z->f) != 56 || fwrite(loc, 1, 20, z->f) != 20 ||
       fwrite(eocd, 1, 22, z->f) != 22 ) return DISCO_ERR_IO;
   return DISCO_OK;
}

int disco_npz_close(disco_npz *z){
   if( !z ) return DISCO_ERR_ARG;
   int s = DISCO_OK;
   if( z->writing ){
      if( z->open ) s = DISCO_ERR_ARG;         /* a member left unfinished */
      else s = write_directory(z);
   }
   if( fclose(z->f) != 0 && !s ) s = DISCO_ERR_IO;
   int n = z->nmem + (z->writing && z->open ? 1 : 0);
   for( int i=0 ; i<n ; ++i ) free(z->mem[i].name);
   free(z);
   return s;
}

/* ------------------------------------------------------------ reading */

static int read_at(FILE *f, uint64_t off, void *dst, size_t n){
   if( fseeko(f, (off_t)off, SEEK_SET) ) return 1;
   return fread(dst, 1, n, f) != n;
}

static int read_directory(disco_npz *z){
   FILE *f = z->f;
   if( fseeko(f, 0, SEEK_END) ) return DISCO_ERR_IO;
   uint64_t fsize = (uint64_t)ftello(f);
   if( fsize < 22 ) return DISCO_ERR_IO;
   size_t tail = fsize < 65557 ? (size_t)fsize : 65557;
   unsigned char *t = (unsigned char *)malloc(tail);
   if( !t ) return DISCO_ERR_IO;
   if( read_at(f, fsize - tail, t, tail) ){ free(t); return DISCO_ERR_IO; }
   long e = -1;
   for( long p=(long)tail-22 ; p>=0 ; --p ) if( get32(t + p) == 0x06054b50u ){ e = p; break; }
   if( e < 0 ){ free(t); return DISCO_ERR_IO; }
   uint64_t eocd_pos = fsize - tail + (uint64_t)e;
   uint64_t nent = get16(t + e + 10), cd_size = get32(t + e + 12), cd_off = get32(t + e + 16);
   free(t);
   if( eocd_pos >= 20 + 56 ){
      unsigned char loc[20];
      if( !read_at(f, eocd_pos - 20, loc, 20) && get32(loc) == 0x07064b50u ){
         unsigned char e64[56];
         if( read_at(f, get64(loc + 8), e64, 56) || get32(e64) != 0x06064b50u ) return DISCO_ERR_IO;
         nent = get64(e64 + 32); cd_size = get64(e64 + 40); cd_off = get64(e64 + 48);
      }
   }
   if( nent > NPZ_MAXMEM || cd_off + cd_size > fsize ) return DISCO_ERR_IO;
   unsigned char *cd = (unsigned char *)malloc(cd_size ? cd_size : 1);
   if( !cd ) return DISCO_ERR_IO;
   if( read_at(f, cd_off, cd, cd_size) ){ free(cd); return DISCO_ERR_IO; }
   uint64_t p = 0;
   for( uint64_t i=0 ; i<nent ; ++i ){
      if( p + 46 > cd_size || get32(cd + p) != 0x02014b50u ){ free(cd); return DISCO_ERR_IO; }
      unsigned method = get16(cd + p + 10);
      uint32_t crc = get32(cd + p + 16);
      uint64_t csize = get32(cd + p + 20), usize = get32(cd + p + 24);
      unsigned nl = get16(cd + p + 28), xl = get16(cd + p + 30), kl = get16(cd + p + 32);
      uint64_t off = get32(cd + p + 42);
      if( p + 46 + nl + xl + kl > cd_size ){ free(cd); return DISCO_ERR_IO; }
      /* ZIP64 extra: the fields whose 32-bit value is saturated, in order */
      const unsigned char *x = cd + p + 46 + nl, *xe = x + xl;
      while( x + 4 <= xe ){
         unsigned id = get16(x), sz = get16(x + 2);
         const unsigned char *v = x + 4, *ve = v + sz;
         if( ve > xe ) break;
         if( id == 1 ){
            if( usize == 0xffffffffu && v + 8 <= ve ){ usize = get64(v); v += 8; }
            if( csize == 0xffffffffu && v + 8 <= ve ){ csize = get64(v); v += 8; }
            if( off == 0xffffffffu && v + 8 <= ve ){ off = get64(v); v += 8; }
         }
         x = ve;
      }
      struct npz_member *m = &z->mem[z->nmem];
      m->name = (char *)malloc(nl + 1);
      if( !m->name ){ free(cd); return DISCO_ERR_IO; }
      memcpy(m->name, cd + p + 46, nl);
      m->name[nl] = '\0';
      m->offset = off;
      m->size = method == 0 && csize == usize ? usize : UINT64_MAX;   /* compressed: refused on read */
      m->crc = crc;
      m->data_off = 0;
      z->nmem++;
      p += 46 + nl + xl + kl;
   }
   free(cd);
   return DISCO_OK;
}

int disco_npz_open(const char *path, disco_npz **out){
   if( !path || !out ) return DISCO_ERR_ARG;
   *out = NULL;
   disco_npz *z = (disco_npz *)calloc(1, sizeof *z);
   if( !z ) return DISCO_ERR_IO;
   z->f = fopen(path, "rb");
   if( !z->f ){ free(z); return DISCO_ERR_IO; }
   int s = read_directory(z);
   if( s ){ disco_npz_close(z); return s; }
   *out = z;
   return DISCO_OK;
}

static struct npz_member *find(disco_npz *z, const char *name){
   char fname[600];
   snprintf(fname, sizeof fname, "%s.npy", name);
   for( int i=0 ; i<z->nmem ; ++i ) if( strcmp(z->mem[i].name, fname) == 0 ) return &z->mem[i];
   return NULL;
}

/* parse the member's .npy header: descr, shape; sets m->data_off */
static int parse_npy(disco_npz *z, struct npz_member *m, char *descr, int *ndim, int64_t *shape){
   if( m->size == UINT64_MAX ) return DISCO_ERR_UNSUPPORTED;      /* compressed member */
   unsigned char lh[30];
   if( read_at(z->f, m->offset, lh, 30) || get32(lh) != 0x04034b50u ) return DISCO_ERR_IO;
   uint64_t start = m->offset + 30 + get16(lh + 26) + get16(lh + 28);
   unsigned char pre[12];
   if( read_at(z->f, start, pre, 12) || memcmp(pre, "\x93NUMPY", 6) ) return DISCO_ERR_IO;
   uint64_t hlen, hoff;
   if( pre[6] == 1 ){ hlen = get16(pre + 8); hoff = 10; }
   else { hlen = get32(pre + 8); hoff = 12; }
   if( hlen > 65536 || hoff + hlen > m->size ) return DISCO_ERR_IO;
   char *h = (char *)malloc((size_t)hlen + 1);
   if( !h ) return DISCO_ERR_IO;
   if( read_at(z->f, start + hoff, h, hlen) ){ free(h); return DISCO_ERR_IO; }
   h[hlen] = '\0';
   int s = DISCO_OK;
   char *d = strstr(h, "'descr':"), *fo = strstr(h, "'fortran_order':"), *sh = strstr(h, "'shape':");
   if( !d || !fo || !sh ) s = DISCO_ERR_IO;
   if( !s ){
      d = strchr(d + 8, '\'');
      char *de = d ? strchr(d + 1, '\'') : NULL;
      if( !d || !de || de - d - 1 >= 16 ) s = DISCO_ERR_IO;
      else { memcpy(descr, d + 1, de - d - 1); descr[de - d - 1] = '\0'; }
   }
   if( !s && strncmp(fo + 16 + strspn(fo + 16, " "), "False", 5) ) s = DISCO_ERR_UNSUPPORTED;
   if( !s ){
      char *p = strchr(sh, '(');
      int n = 0;
      if( !p ) s = DISCO_ERR_IO;
      else {
         ++p;
         while( !s ){
            p += strspn(p, " ,");
            if( *p == ')' ) break;
            char *q;
            long long v = strtoll(p, &q, 10);
            if( q == p || n >= 8 ) s = DISCO_ERR_IO;
            else { shape[n++] = v; p = q; }
         }
      }
      *ndim = n;
   }
   free(h);
   if( !s ){
      int isz = itemsize(descr);
      uint64_t count = 1;
      for( int i=0 ; i<*ndim ; ++i ) count *= (uint64_t)shape[i];
      if( isz <= 0 || hoff + hlen + count*(uint64_t)isz != m->size ) s = DISCO_ERR_IO;
      m->data_off = start + hoff + hlen;
      m->data_bytes = count*(uint64_t)isz;
   }
   return s;
}

int disco_npz_info(disco_npz *z, const char *name, char *descr, int *ndim, int64_t *shape){
   if( !z || z->writing || !name || !descr || !ndim || !shape ) return DISCO_ERR_ARG;
   struct npz_member *m = find(z, name);
   if( !m ) return DISCO_ERR_IO;
   return parse_npy(z, m, descr, ndim, shape);
}

int disco_npz_read(disco_npz *z, const char *name, uint64_t offset, void *dst, size_t nbytes){
   if( !z || z->writing || !name || (!dst && nbytes) ) return DISCO_ERR_ARG;
   struct npz_member *m = find(z, name);
   if( !m ) return DISCO_ERR_IO;
   char descr[16];
   int ndim;
   int64_t shape[8];
   int s = parse_npy(z, m, descr, &ndim, shape);
   if( s ) return s;
   if( offset > m->data_bytes || nbytes > m->data_bytes - offset ) return DISCO_ERR_ARG;
   if( nbytes && read_at(z->f, m->data_off + offset, dst, nbytes) ) return DISCO_ERR_IO;
   return DISCO_OK;
}
