/*
 * GSList subset of glib-2.0 (see glib.h in this folder).
 * TEST INFRASTRUCTURE ONLY.
 */
#include "glib.h"

#include <stdlib.h>

GSList *g_slist_alloc(void) { return (GSList *)calloc(1, sizeof(GSList)); }

void g_slist_free_1(GSList *list) { free(list); }

void g_slist_free(GSList *list)
{
    while (list) {
        GSList *next = list->next;
        free(list);
        list = next;
    }
}

GSList *g_slist_remove_link(GSList *list, GSList *link_)
{
    GSList *prev = NULL, *cur = list;
    while (cur) {
        if (cur == link_) {
            if (prev)
                prev->next = cur->next;
            else
                list = cur->next;
            cur->next = NULL;
            break;
        }
        prev = cur;
        cur = cur->next;
    }
    return list;
}

guint g_slist_length(GSList *list)
{
    guint n = 0;
    for (; list; list = list->next)
        n++;
    return n;
}

void g_slist_foreach(GSList *list, GFunc func, gpointer user_data)
{
    while (list) {
        GSList *next = list->next;
        func(list->data, user_data);
        list = next;
    }
}

GSList *g_slist_prepend(GSList *list, gpointer data)
{
    GSList *node = g_slist_alloc();
    node->data = data;
    node->next = list;
    return node;
}

GSList *g_slist_append(GSList *list, gpointer data)
{
    GSList *node = g_slist_alloc(), *last = list;
    node->data = data;
    if (!list)
        return node;
    while (last->next)
        last = last->next;
    last->next = node;
    return list;
}

GSList *g_slist_reverse(GSList *list)
{
    GSList *prev = NULL;
    while (list) {
        GSList *next = list->next;
        list->next = prev;
        prev = list;
        list = next;
    }
    return prev;
}

GSList *g_slist_nth(GSList *list, guint n)
{
    while (n-- > 0 && list)
        list = list->next;
    return list;
}

/* Stable merge sort, as glib's g_slist_sort is documented to be. */
static GSList *merge(GSList *a, GSList *b, GCompareFunc cmp)
{
    GSList head, *tail = &head;
    while (a && b) {
        if (cmp(a->data, b->data) <= 0) {
            tail->next = a;
            a = a->next;
        } else {
            tail->next = b;
            b = b->next;
        }
        tail = tail->next;
    }
    tail->next = a ? a : b;
    return head.next;
}

GSList *g_slist_sort(GSList *list, GCompareFunc compare_func)
{
    GSList *slow, *fast, *second;
    if (!list || !list->next)
        return list;
    slow = list;
    fast = list->next;
    while (fast && fast->next) {
        slow = slow->next;
        fast = fast->next->next;
    }
    second = slow->next;
    slow->next = NULL;
    return merge(g_slist_sort(list, compare_func), g_slist_sort(second, compare_func),
                 compare_func);
}
