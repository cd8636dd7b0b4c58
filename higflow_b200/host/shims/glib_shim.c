/*
 * Chained hash table implementing the GLib subset declared in glib.h.
 * Oracle build only (test infrastructure).
 */
#include "glib.h"

#include <stdio.h>
#include <string.h>

typedef struct node {
    gpointer key;
    gpointer value;
    struct node *next;
} node;

struct _GHashTable {
    GHashFunc hash;
    GEqualFunc equal;
    GDestroyNotify key_destroy;
    GDestroyNotify value_destroy;
    node **buckets;
    size_t nbuckets;
    size_t count;
};

guint g_direct_hash(gconstpointer v)
{
    uintptr_t x = (uintptr_t)v;
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    return (guint)x;
}

gboolean g_direct_equal(gconstpointer a, gconstpointer b) { return a == b; }

static void oom(void)
{
    fprintf(stderr, "glib shim: out of memory\n");
    abort();
}

GHashTable *g_hash_table_new_full(GHashFunc hash, GEqualFunc equal,
                                  GDestroyNotify key_destroy,
                                  GDestroyNotify value_destroy)
{
    GHashTable *t = calloc(1, sizeof *t);
    if (!t) oom();
    t->hash = hash ? hash : g_direct_hash;
    t->equal = equal ? equal : g_direct_equal;
    t->key_destroy = key_destroy;
    t->value_destroy = value_destroy;
    t->nbuckets = 64;
    t->buckets = calloc(t->nbuckets, sizeof(node *));
    if (!t->buckets) oom();
    return t;
}

GHashTable *g_hash_table_new(GHashFunc hash, GEqualFunc equal)
{
    return g_hash_table_new_full(hash, equal, NULL, NULL);
}

static node **find(GHashTable *t, gconstpointer key)
{
    size_t b = t->hash(key) % t->nbuckets;
    node **pp = &t->buckets[b];
    while (*pp) {
        if (t->equal((*pp)->key, key)) return pp;
        pp = &(*pp)->next;
    }
    return pp;
}

static void grow(GHashTable *t)
{
    size_t nb = t->nbuckets * 4;
    node **nbk = calloc(nb, sizeof(node *));
    if (!nbk) oom();
    for (size_t i = 0; i < t->nbuckets; i++) {
        node *n = t->buckets[i];
        while (n) {
            node *nx = n->next;
            size_t b = t->hash(n->key) % nb;
            n->next = nbk[b];
            nbk[b] = n;
            n = nx;
        }
    }
    free(t->buckets);
    t->buckets = nbk;
    t->nbuckets = nb;
}

gboolean g_hash_table_insert(GHashTable *t, gpointer key, gpointer value)
{
    node **pp = find(t, key);
    if (*pp) {
        /* GLib keeps the original key, drops the new one, replaces the value. */
        if (t->key_destroy) t->key_destroy(key);
        if (t->value_destroy) t->value_destroy((*pp)->value);
        (*pp)->value = value;
        return FALSE;
    }
    node *n = malloc(sizeof *n);
    if (!n) oom();
    n->key = key;
    n->value = value;
    n->next = NULL;
    *pp = n;
    t->count++;
    if (t->count > 2 * t->nbuckets) grow(t);
    return TRUE;
}

gpointer g_hash_table_lookup(GHashTable *t, gconstpointer key)
{
    node **pp = find(t, key);
    return *pp ? (*pp)->value : NULL;
}

gboolean g_hash_table_lookup_extended(GHashTable *t, gconstpointer key,
                                      gpointer *orig_key, gpointer *value)
{
    node **pp = find(t, key);
    if (!*pp) return FALSE;
    if (orig_key) *orig_key = (*pp)->key;
    if (value) *value = (*pp)->value;
    return TRUE;
}

gboolean g_hash_table_contains(GHashTable *t, gconstpointer key)
{
    return *find(t, key) != NULL;
}

gboolean g_hash_table_remove(GHashTable *t, gconstpointer key)
{
    node **pp = find(t, key);
    if (!*pp) return FALSE;
    node *n = *pp;
    *pp = n->next;
    if (t->key_destroy) t->key_destroy(n->key);
    if (t->value_destroy) t->value_destroy(n->value);
    free(n);
    t->count--;
    return TRUE;
}

void g_hash_table_remove_all(GHashTable *t)
{
    for (size_t i = 0; i < t->nbuckets; i++) {
        node *n = t->buckets[i];
        while (n) {
            node *nx = n->next;
            if (t->key_destroy) t->key_destroy(n->key);
            if (t->value_destroy) t->value_destroy(n->value);
            free(n);
            n = nx;
        }
        t->buckets[i] = NULL;
    }
    t->count = 0;
}

guint g_hash_table_size(GHashTable *t) { return (guint)t->count; }

void g_hash_table_destroy(GHashTable *t)
{
    if (!t) return;
    g_hash_table_remove_all(t);
    free(t->buckets);
    free(t);
}

void g_hash_table_iter_init(GHashTableIter *it, GHashTable *t)
{
    it->table = t;
    it->bucket = 0;
    it->node = NULL;
    it->next = NULL;
    while (it->bucket < t->nbuckets && !t->buckets[it->bucket]) it->bucket++;
    if (it->bucket < t->nbuckets) it->next = t->buckets[it->bucket];
}

gboolean g_hash_table_iter_next(GHashTableIter *it, gpointer *key, gpointer *value)
{
    GHashTable *t = it->table;
    node *n = it->next;
    if (!n) return FALSE;
    if (key) *key = n->key;
    if (value) *value = n->value;
    if (n->next) {
        it->next = n->next;
    } else {
        it->bucket++;
        while (it->bucket < t->nbuckets && !t->buckets[it->bucket]) it->bucket++;
        it->next = it->bucket < t->nbuckets ? t->buckets[it->bucket] : NULL;
    }
    it->node = n;
    return TRUE;
}
