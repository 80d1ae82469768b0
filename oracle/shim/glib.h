/*
 * Stand-in for the subset of glib-2.0 that the reference accelsearch sources
 * call (singly-linked GSList only).  glib is not installed in this image, so
 * the oracle's reference build links against this header and glib_shim.c.
 * Semantics follow glib's published documentation for these functions.
 *
 * TEST INFRASTRUCTURE ONLY: nothing in the product library includes this.
 */
#ifndef ORACLE_SHIM_GLIB_H
#define ORACLE_SHIM_GLIB_H

#ifdef __cplusplus
extern "C" {
#endif

typedef void *gpointer;
typedef const void *gconstpointer;
typedef int gint;
typedef unsigned int guint;
typedef int gboolean;
typedef gint (*GCompareFunc)(gconstpointer a, gconstpointer b);
typedef void (*GFunc)(gpointer data, gpointer user_data);

typedef struct _GSList GSList;
struct _GSList {
    gpointer data;
    GSList *next;
};

GSList *g_slist_alloc(void);
void g_slist_free_1(GSList *list);
void g_slist_free(GSList *list);
GSList *g_slist_remove_link(GSList *list, GSList *link_);
GSList *g_slist_sort(GSList *list, GCompareFunc compare_func);
guint g_slist_length(GSList *list);
void g_slist_foreach(GSList *list, GFunc func, gpointer user_data);
GSList *g_slist_append(GSList *list, gpointer data);
GSList *g_slist_prepend(GSList *list, gpointer data);
GSList *g_slist_reverse(GSList *list);
GSList *g_slist_nth(GSList *list, guint n);

#ifdef __cplusplus
}
#endif

#endif
