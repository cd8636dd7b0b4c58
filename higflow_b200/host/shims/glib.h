/*
 * Minimal GLib stand-in for building the reference HigTree/HigFlow C sources
 * in place in this image, which has no GLib (the HigFlow host build,
 * higflow_b200/host, and the oracle build of the reference).
 *
 * Only the GHashTable surface that higtree/src/{mapper,point-mapper,pdomain,
 * mapper-syncer}.c use is provided: a chained hash table with the GLib
 * semantics those files rely on (direct hashing of pointer-sized keys when the
 * hash function is NULL, key/value destroy notifiers, insert-replaces-value,
 * lookup_extended).  Iteration order is unspecified, as in GLib; on one rank
 * the reference never iterates a non-empty table on the step path.
 */
#ifndef HF_ORACLE_GLIB_SHIM_H
#define HF_ORACLE_GLIB_SHIM_H

#include <float.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>

#define GLIB_CHECK_VERSION(major, minor, micro) 1

typedef void *gpointer;
typedef const void *gconstpointer;
typedef unsigned int guint;
typedef int gint;
typedef int gboolean;
typedef size_t gsize;

#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif

typedef guint (*GHashFunc)(gconstpointer key);
typedef gboolean (*GEqualFunc)(gconstpointer a, gconstpointer b);
typedef void (*GDestroyNotify)(gpointer data);

typedef struct _GHashTable GHashTable;

typedef struct _GHashTableIter {
    GHashTable *table;
    size_t bucket;
    void *node;
    void *next;
} GHashTableIter;

#define GINT_TO_POINTER(i) ((gpointer)(intptr_t)(i))
#define GPOINTER_TO_INT(p) ((gint)(intptr_t)(p))
#define GUINT_TO_POINTER(u) ((gpointer)(uintptr_t)(u))
#define GPOINTER_TO_UINT(p) ((guint)(uintptr_t)(p))

#define g_new(type, n) ((type *)malloc(sizeof(type) * (size_t)(n)))

guint g_direct_hash(gconstpointer v);
gboolean g_direct_equal(gconstpointer a, gconstpointer b);

GHashTable *g_hash_table_new(GHashFunc hash, GEqualFunc equal);
GHashTable *g_hash_table_new_full(GHashFunc hash, GEqualFunc equal,
                                  GDestroyNotify key_destroy,
                                  GDestroyNotify value_destroy);
gboolean g_hash_table_insert(GHashTable *t, gpointer key, gpointer value);
gpointer g_hash_table_lookup(GHashTable *t, gconstpointer key);
gboolean g_hash_table_lookup_extended(GHashTable *t, gconstpointer key,
                                      gpointer *orig_key, gpointer *value);
gboolean g_hash_table_contains(GHashTable *t, gconstpointer key);
gboolean g_hash_table_remove(GHashTable *t, gconstpointer key);
void g_hash_table_remove_all(GHashTable *t);
guint g_hash_table_size(GHashTable *t);
void g_hash_table_destroy(GHashTable *t);
void g_hash_table_iter_init(GHashTableIter *it, GHashTable *t);
gboolean g_hash_table_iter_next(GHashTableIter *it, gpointer *key, gpointer *value);

#endif
