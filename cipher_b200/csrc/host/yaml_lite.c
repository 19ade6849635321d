/*
 * yaml_lite.c - parser for the YAML subset of the configuration files and
 * the reference's GetProperty lookup on its event stream (src/init.c:24-99).
 */
#define _POSIX_C_SOURCE 200809L
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "yaml_lite.h"

typedef struct {
    const char *s;               /* line text, no line end */
    int len;
    int indent;                  /* leading spaces */
    int lineno;
} yl_line;

typedef struct {
    yl_line *L;
    int n, i;
    char *err;
    size_t errlen;
    int failed;
} yl_parser;

static void fail(yl_parser *p, int lineno, const char *fmt, ...)
{
    if (p->failed) return;
    p->failed = 1;
    if (!p->err || !p->errlen) return;
    int k = snprintf(p->err, p->errlen, "line %d: ", lineno);
    if (k < 0 || (size_t)k >= p->errlen) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(p->err + k, p->errlen - (size_t)k, fmt, ap);
    va_end(ap);
}

/* ---------------- nodes ---------------- */

static char *dupn(const char *s, size_t n)
{
    char *d = (char *)malloc(n + 1);
    if (!d) return NULL;
    memcpy(d, s, n);
    d[n] = 0;
    return d;
}

static yl_node *node_new(int kind)
{
    yl_node *n = (yl_node *)calloc(1, sizeof(yl_node));
    if (n) n->kind = kind;
    return n;
}

static yl_node *scalar_new(const char *s, size_t len)
{
    yl_node *n = node_new(YL_SCALAR);
    if (n) n->value = dupn(s, len);
    if (n && !n->value) { free(n); return NULL; }
    return n;
}

static void node_free(yl_node *n)
{
    if (!n) return;
    free(n->value);
    for (int i = 0; i < n->n; i++) {
        if (n->keys) free(n->keys[i]);
        node_free(n->kids[i]);
    }
    free(n->keys);
    free(n->kids);
    free(n);
}

static int node_add(yl_node *n, char *key, yl_node *kid)
{
    if (n->n == n->cap) {
        int cap = n->cap ? 2 * n->cap : 8;
        yl_node **k = (yl_node **)realloc(n->kids, (size_t)cap * sizeof(yl_node *));
        if (!k) return 1;
        n->kids = k;
        if (n->kind == YL_MAPPING) {
            char **ks = (char **)realloc(n->keys, (size_t)cap * sizeof(char *));
            if (!ks) return 1;
            n->keys = ks;
        }
        n->cap = cap;
    }
    if (n->kind == YL_MAPPING) n->keys[n->n] = key;
    n->kids[n->n++] = kid;
    return 0;
}

/* ---------------- lines ---------------- */

static int is_blank(const yl_line *l)
{
    for (int k = 0; k < l->len; k++)
        if (l->s[k] != ' ' && l->s[k] != '\t') return 0;
    return 1;
}

/* a line with no content for block structure: blank or a comment */
static int is_void(const yl_line *l)
{
    if (is_blank(l)) return 1;
    return l->s[l->indent] == '#';
}

static int next_content(yl_parser *p)
{
    while (p->i < p->n && is_void(&p->L[p->i])) p->i++;
    return p->i < p->n ? p->i : -1;
}

/* [b, e) without surrounding blanks */
static void trim(const char *s, int *b, int *e)
{
    while (*b < *e && (s[*b] == ' ' || s[*b] == '\t')) (*b)++;
    while (*e > *b && (s[*e - 1] == ' ' || s[*e - 1] == '\t')) (*e)--;
}

/* end of the text before a comment: '#' at the start or after a blank,
 * outside quotes */
static int comment_start(const char *s, int b, int e)
{
    char q = 0;
    for (int k = b; k < e; k++) {
        const char c = s[k];
        if (q) {
            if (c == q) {
                if (q == '\'' && k + 1 < e && s[k + 1] == '\'') { k++; continue; }
                q = 0;
            } else if (q == '"' && c == '\\') k++;
        } else if (c == '"' || c == '\'') {
            if (k == b || s[k - 1] == ' ' || s[k - 1] == '\t' || s[k - 1] == '[' || s[k - 1] == ',' ||
                s[k - 1] == '{' || s[k - 1] == ':')
                q = c;
        } else if (c == '#' && (k == b || s[k - 1] == ' ' || s[k - 1] == '\t')) {
            return k;
        }
    }
    return e;
}

/* position of the mapping separator ':' (followed by a blank or the end of
 * the text), outside quotes and brackets, or -1 */
static int key_colon(const char *s, int b, int e)
{
    char q = 0;
    int depth = 0;
    for (int k = b; k < e; k++) {
        const char c = s[k];
        if (q) {
            if (c == q) q = 0;
            else if (q == '"' && c == '\\') k++;
            continue;
        }
        if ((c == '"' || c == '\'') && k == b) { q = c; continue; }
        if (c == '[' || c == '{') depth++;
        else if (c == ']' || c == '}') depth--;
        else if (c == ':' && depth == 0 && (k + 1 == e || s[k + 1] == ' ' || s[k + 1] == '\t')) return k;
    }
    return -1;
}

/* quoted scalar at s[b..e) (s[b] is the quote) into a new string; *end =
 * one past the closing quote */
static char *unquote(yl_parser *p, int lineno, const char *s, int b, int e, int *end)
{
    const char q = s[b];
    char *out = (char *)malloc((size_t)(e - b) + 1);
    if (!out) return NULL;
    int o = 0, k = b + 1;
    for (; k < e; k++) {
        const char c = s[k];
        if (c == q) {
            if (q == '\'' && k + 1 < e && s[k + 1] == '\'') { out[o++] = '\''; k++; continue; }
            break;
        }
        if (q == '"' && c == '\\' && k + 1 < e) {
            const char x = s[++k];
            out[o++] = x == 'n' ? '\n' : x == 't' ? '\t' : x == '0' ? '\0' : x;
            continue;
        }
        out[o++] = c;
    }
    if (k >= e) {
        free(out);
        fail(p, lineno, "unterminated quoted scalar");
        return NULL;
    }
    out[o] = 0;
    *end = k + 1;
    return out;
}

/* ---------------- flow collections ---------------- */

static yl_node *flow_node(yl_parser *p, int lineno, const char *s, int *k, int e);

static void skip_ws(const char *s, int *k, int e)
{
    while (*k < e && (s[*k] == ' ' || s[*k] == '\t' || s[*k] == '\n')) (*k)++;
}

/* a plain scalar inside a flow collection: up to ',' ']' '}' (and ": " for
 * a key) */
static yl_node *flow_scalar(yl_parser *p, int lineno, const char *s, int *k, int e, int key)
{
    skip_ws(s, k, e);
    if (*k < e && (s[*k] == '"' || s[*k] == '\'')) {
        int end;
        char *v = unquote(p, lineno, s, *k, e, &end);
        if (!v) return NULL;
        *k = end;
        yl_node *n = node_new(YL_SCALAR);
        if (!n) { free(v); return NULL; }
        n->value = v;
        return n;
    }
    int b = *k;
    while (*k < e) {
        const char c = s[*k];
        if (c == ',' || c == ']' || c == '}') break;
        if (key && c == ':' && (*k + 1 == e || s[*k + 1] == ' ' || s[*k + 1] == ',' || s[*k + 1] == '}')) break;
        if (c == '[' || c == '{') { fail(p, lineno, "unexpected '%c' in a flow scalar", c); return NULL; }
        (*k)++;
    }
    int ee = *k;
    trim(s, &b, &ee);
    /* a line break inside a flow scalar folds to one space */
    char *v = dupn(s + b, (size_t)(ee - b));
    if (!v) return NULL;
    for (char *c = v; *c; c++)
        if (*c == '\n') *c = ' ';
    yl_node *n = node_new(YL_SCALAR);
    if (!n) { free(v); return NULL; }
    n->value = v;
    return n;
}

static yl_node *flow_node(yl_parser *p, int lineno, const char *s, int *k, int e)
{
    skip_ws(s, k, e);
    if (*k >= e) { fail(p, lineno, "unexpected end of a flow collection"); return NULL; }
    const char open = s[*k];
    if (open != '[' && open != '{') return flow_scalar(p, lineno, s, k, e, 0);
    const char close = open == '[' ? ']' : '}';
    yl_node *n = node_new(open == '[' ? YL_SEQUENCE : YL_MAPPING);
    if (!n) return NULL;
    (*k)++;
    for (;;) {
        skip_ws(s, k, e);
        if (*k >= e) { fail(p, lineno, "unterminated flow collection"); node_free(n); return NULL; }
        if (s[*k] == close) { (*k)++; return n; }
        char *key = NULL;
        yl_node *kid;
        if (n->kind == YL_MAPPING) {
            yl_node *kn = flow_scalar(p, lineno, s, k, e, 1);
            if (!kn) { node_free(n); return NULL; }
            key = kn->value;
            kn->value = NULL;
            node_free(kn);
            skip_ws(s, k, e);
            if (*k < e && s[*k] == ':') {
                (*k)++;
                skip_ws(s, k, e);
                if (*k < e && (s[*k] == ',' || s[*k] == close)) kid = scalar_new("", 0);
                else kid = flow_node(p, lineno, s, k, e);
            } else {
                kid = scalar_new("", 0);
            }
        } else {
            kid = flow_node(p, lineno, s, k, e);
        }
        if (!kid || node_add(n, key, kid)) { free(key); node_free(kid); node_free(n); return NULL; }
        skip_ws(s, k, e);
        if (*k < e && s[*k] == ',') { (*k)++; continue; }
        if (*k < e && s[*k] == close) continue;
        fail(p, lineno, "expected ',' or '%c' in a flow collection", close);
        node_free(n);
        return NULL;
    }
}

/* a flow collection that starts in `rest` and may continue on later lines */
static yl_node *flow_value(yl_parser *p, int lineno, const char *s, int b, int e)
{
    /* gather text until the brackets balance, comments removed */
    size_t cap = (size_t)(e - b) + 2, len = 0;
    char *buf = (char *)malloc(cap);
    if (!buf) return NULL;
    int depth = 0;
    char q = 0;
    const char *ls = s;
    int lb = b, le = e;
    for (;;) {
        le = comment_start(ls, lb, le);
        for (int k = lb; k < le; k++) {
            const char c = ls[k];
            if (q) {
                if (q == '"' && c == '\\') k++;
                else if (c == q) q = 0;
            }
            else if (c == '"' || c == '\'') q = c;
            else if (c == '[' || c == '{') depth++;
            else if (c == ']' || c == '}') depth--;
        }
        if (len + (size_t)(le - lb) + 2 > cap) {
            cap = 2 * (len + (size_t)(le - lb) + 2);
            char *nb = (char *)realloc(buf, cap);
            if (!nb) { free(buf); return NULL; }
            buf = nb;
        }
        memcpy(buf + len, ls + lb, (size_t)(le - lb));
        len += (size_t)(le - lb);
        if (depth <= 0) break;
        buf[len++] = '\n';
        if (p->i >= p->n) { free(buf); fail(p, lineno, "unterminated flow collection"); return NULL; }
        const yl_line *l = &p->L[p->i++];
        ls = l->s;
        lb = 0;
        le = l->len;
    }
    buf[len] = 0;
    int k = 0;
    yl_node *n = flow_node(p, lineno, buf, &k, (int)len);
    if (n) {
        skip_ws(buf, &k, (int)len);
        if (k != (int)len) { fail(p, lineno, "text after a flow collection"); node_free(n); n = NULL; }
    }
    free(buf);
    return n;
}

/* ---------------- block structure ---------------- */

static yl_node *block_node(yl_parser *p, int min_indent);

/* literal ('|') or folded ('>') block scalar whose header is s[b..e);
 * `ind` is the indentation of the owning key or item */
static yl_node *block_scalar(yl_parser *p, int lineno, const char *s, int b, int e, int ind)
{
    const char style = s[b];
    int chomp = 0, explicit_ind = 0;
    for (int k = b + 1; k < e; k++) {
        if (s[k] == '-') chomp = -1;
        else if (s[k] == '+') chomp = 1;
        else if (s[k] >= '1' && s[k] <= '9') explicit_ind = s[k] - '0';
        else if (s[k] == ' ' || s[k] == '\t') { if (comment_start(s, k, e) == k) break; }
        else if (s[k] == '#') break;
        else { fail(p, lineno, "bad block scalar header"); return NULL; }
    }
    int cind = explicit_ind ? ind + explicit_ind : -1;
    if (cind < 0) {
        for (int j = p->i; j < p->n; j++)
            if (!is_blank(&p->L[j])) { cind = p->L[j].indent; break; }
        if (cind <= ind) cind = ind + 1;  /* empty scalar */
    }
    size_t cap = 64, len = 0;
    char *buf = (char *)malloc(cap);
    if (!buf) return NULL;
    int nl_pending = 0;          /* folded: line breaks since the last text */
    int first = 1;
    while (p->i < p->n) {
        const yl_line *l = &p->L[p->i];
        if (!is_blank(l) && l->indent < cind) break;
        p->i++;
        const char *t = l->len > cind ? l->s + cind : "";
        const size_t tl = l->len > cind ? (size_t)(l->len - cind) : 0;
        const size_t need = len + tl + (size_t)nl_pending + 2;
        if (need > cap) {
            cap = 2 * need;
            char *nb = (char *)realloc(buf, cap);
            if (!nb) { free(buf); return NULL; }
            buf = nb;
        }
        if (style == '|') {
            memcpy(buf + len, t, tl);
            len += tl;
            buf[len++] = '\n';
        } else {
            if (is_blank(l)) { nl_pending++; continue; }
            if (!first) {
                if (nl_pending) while (nl_pending--) buf[len++] = '\n';
                else buf[len++] = ' ';
            }
            nl_pending = 0;
            memcpy(buf + len, t, tl);
            len += tl;
            first = 0;
        }
    }
    if (style == '>') {
        if (!first) buf[len++] = '\n';
        for (int k = 0; k < nl_pending; k++) {
            if (len + 2 > cap) {
                cap *= 2;
                char *nb = (char *)realloc(buf, cap);
                if (!nb) { free(buf); return NULL; }
                buf = nb;
            }
            buf[len++] = '\n';
        }
    }
    /* chomping: strip (-) no final line break, clip one, keep (+) all */
    if (chomp <= 0) {
        while (len > 0 && buf[len - 1] == '\n') len--;
        if (chomp == 0 && len > 0) buf[len++] = '\n';
    }
    yl_node *n = node_new(YL_SCALAR);
    if (!n) { free(buf); return NULL; }
    buf[len] = 0;
    n->value = buf;
    return n;
}

/* the value after "key:" (or "- "): rest = s[b..e) on the key's line */
static yl_node *value_node(yl_parser *p, int lineno, const char *s, int b, int e, int ind)
{
    e = comment_start(s, b, e);
    trim(s, &b, &e);
    if (b == e) {
        const int j = next_content(p);
        if (j >= 0 && p->L[j].indent > ind) return block_node(p, ind + 1);
        if (j >= 0 && p->L[j].indent == ind && p->L[j].s[ind] == '-' &&
            (p->L[j].len == ind + 1 || p->L[j].s[ind + 1] == ' '))
            return block_node(p, ind);              /* "key:\n- a" at the key's indentation */
        return scalar_new("", 0);
    }
    const char c = s[b];
    if (c == '|' || c == '>') return block_scalar(p, lineno, s, b, e, ind);
    if (c == '[' || c == '{') return flow_value(p, lineno, s, b, e);
    if (c == '&' || c == '*' || c == '!') { fail(p, lineno, "anchors, aliases and tags are not supported"); return NULL; }
    if (c == '"' || c == '\'') {
        int end;
        char *v = unquote(p, lineno, s, b, e, &end);
        if (!v) return NULL;
        int ee = e, bb = end;
        trim(s, &bb, &ee);
        if (bb != ee) { free(v); fail(p, lineno, "text after a quoted scalar"); return NULL; }
        yl_node *n = node_new(YL_SCALAR);
        if (!n) { free(v); return NULL; }
        n->value = v;
        return n;
    }
    if (key_colon(s, b, e) >= 0) { fail(p, lineno, "mapping values are not allowed here"); return NULL; }
    /* plain scalar, continued on more-indented lines (folded with spaces) */
    size_t cap = (size_t)(e - b) + 1, len = (size_t)(e - b);
    char *buf = dupn(s + b, (size_t)(e - b));
    if (!buf) return NULL;
    for (;;) {
        const int j = next_content(p);
        if (j < 0 || p->L[j].indent <= ind) break;
        const yl_line *l = &p->L[j];
        int lb = l->indent, le = comment_start(l->s, l->indent, l->len);
        trim(l->s, &lb, &le);
        if (key_colon(l->s, lb, le) >= 0) { free(buf); fail(p, l->lineno, "mapping values are not allowed here"); return NULL; }
        p->i = j + 1;
        if (len + (size_t)(le - lb) + 2 > cap) {
            cap = 2 * (len + (size_t)(le - lb) + 2);
            char *nb = (char *)realloc(buf, cap);
            if (!nb) { free(buf); return NULL; }
            buf = nb;
        }
        buf[len++] = ' ';
        memcpy(buf + len, l->s + lb, (size_t)(le - lb));
        len += (size_t)(le - lb);
        buf[len] = 0;
    }
    yl_node *n = node_new(YL_SCALAR);
    if (!n) { free(buf); return NULL; }
    n->value = buf;
    return n;
}

static yl_node *block_sequence(yl_parser *p, int ind)
{
    yl_node *n = node_new(YL_SEQUENCE);
    if (!n) return NULL;
    for (;;) {
        const int j = next_content(p);
        if (j < 0 || p->L[j].indent != ind) break;
        const yl_line *l = &p->L[j];
        if (l->s[ind] != '-' || !(l->len == ind + 1 || l->s[ind + 1] == ' ')) break;
        p->i = j + 1;
        /* "- key: value" opens a mapping at the item's content column */
        int b = ind + 1;
        while (b < l->len && l->s[b] == ' ') b++;
        yl_node *kid;
        const int ce = comment_start(l->s, b, l->len);
        if (b < ce && key_colon(l->s, b, ce) >= 0 && l->s[b] != '[' && l->s[b] != '{' && l->s[b] != '"' &&
            l->s[b] != '\'') {
            /* re-read this line as the first line of a mapping indented at b */
            p->i = j;
            yl_line saved = p->L[j];
            p->L[j].indent = b;
            kid = block_node(p, b);
            p->L[j] = saved;
        } else {
            kid = value_node(p, l->lineno, l->s, ind + 1, l->len, ind);
        }
        if (!kid || node_add(n, NULL, kid)) { node_free(kid); node_free(n); return NULL; }
        if (p->failed) { node_free(n); return NULL; }
    }
    return n;
}

static yl_node *block_mapping(yl_parser *p, int ind)
{
    yl_node *n = node_new(YL_MAPPING);
    if (!n) return NULL;
    for (;;) {
        const int j = next_content(p);
        if (j < 0 || p->L[j].indent < ind) break;
        const yl_line *l = &p->L[j];
        if (l->indent > ind) { fail(p, l->lineno, "unexpected indentation"); node_free(n); return NULL; }
        const int ce = comment_start(l->s, ind, l->len);
        const int colon = key_colon(l->s, ind, ce);
        if (colon < 0) {
            if (l->s[ind] == '-') break;     /* a sequence at the same column ends this mapping */
            fail(p, l->lineno, "expected 'key: value'");
            node_free(n);
            return NULL;
        }
        int kb = ind, ke = colon;
        trim(l->s, &kb, &ke);
        char *key;
        if (kb < ke && (l->s[kb] == '"' || l->s[kb] == '\'')) {
            int end;
            key = unquote(p, l->lineno, l->s, kb, ke, &end);
        } else {
            key = dupn(l->s + kb, (size_t)(ke - kb));
        }
        if (!key) { node_free(n); return NULL; }
        p->i = j + 1;
        yl_node *kid = value_node(p, l->lineno, l->s, colon + 1, l->len, ind);
        if (!kid || node_add(n, key, kid)) { free(key); node_free(kid); node_free(n); return NULL; }
        if (p->failed) { node_free(n); return NULL; }
    }
    return n;
}

static yl_node *block_node(yl_parser *p, int min_indent)
{
    const int j = next_content(p);
    if (j < 0 || p->L[j].indent < min_indent) return scalar_new("", 0);
    const yl_line *l = &p->L[j];
    const int ind = l->indent;
    if (l->s[ind] == '-' && (l->len == ind + 1 || l->s[ind + 1] == ' ')) return block_sequence(p, ind);
    const int ce = comment_start(l->s, ind, l->len);
    if (key_colon(l->s, ind, ce) >= 0) return block_mapping(p, ind);
    /* a lone scalar (a document that is one value) */
    p->i = j + 1;
    return value_node(p, l->lineno, l->s, ind, l->len, ind - 1);
}

/* ---------------- events ---------------- */

static int push(yl_doc *d, int type, const char *value)
{
    if (d->nev == d->capev) {
        int cap = d->capev ? 2 * d->capev : 256;
        yl_event *ev = (yl_event *)realloc(d->ev, (size_t)cap * sizeof(yl_event));
        if (!ev) return 1;
        d->ev = ev;
        d->capev = cap;
    }
    d->ev[d->nev].type = type;
    d->ev[d->nev].value = value;
    d->nev++;
    return 0;
}

static int emit(yl_doc *d, const yl_node *n)
{
    if (n->kind == YL_SCALAR) return push(d, YL_EV_SCALAR, n->value);
    const int map = n->kind == YL_MAPPING;
    if (push(d, map ? YL_EV_MAP_START : YL_EV_SEQ_START, NULL)) return 1;
    for (int i = 0; i < n->n; i++) {
        if (map && push(d, YL_EV_SCALAR, n->keys[i])) return 1;
        if (emit(d, n->kids[i])) return 1;
    }
    return push(d, map ? YL_EV_MAP_END : YL_EV_SEQ_END, NULL);
}

/* ---------------- entry points ---------------- */

yl_doc *yl_parse(const char *text, size_t len, char *err, size_t errlen)
{
    if (err && errlen) err[0] = 0;
    yl_parser p;
    memset(&p, 0, sizeof(p));
    p.err = err;
    p.errlen = errlen;
    /* split into lines (LF or CRLF) */
    int cap = 1024;
    p.L = (yl_line *)malloc((size_t)cap * sizeof(yl_line));
    if (!p.L) return NULL;
    size_t k = 0;
    int lineno = 1;
    while (k < len) {
        size_t e = k;
        while (e < len && text[e] != '\n') e++;
        size_t le = e;
        if (le > k && text[le - 1] == '\r') le--;
        if (p.n == cap) {
            cap *= 2;
            yl_line *nl = (yl_line *)realloc(p.L, (size_t)cap * sizeof(yl_line));
            if (!nl) { free(p.L); return NULL; }
            p.L = nl;
        }
        yl_line *l = &p.L[p.n++];
        l->s = text + k;
        l->len = (int)(le - k);
        l->indent = 0;
        while (l->indent < l->len && l->s[l->indent] == ' ') l->indent++;
        l->lineno = lineno++;
        if (l->indent < l->len && l->s[l->indent] == '\t') {
            fail(&p, l->lineno, "tab in indentation");
            free(p.L);
            return NULL;
        }
        k = e + 1;
    }
    /* document markers: "---" opens the one document, "..." ends it */
    int first = next_content(&p);
    if (first >= 0) {
        const yl_line *l = &p.L[first];
        if (l->indent == 0 && l->len >= 3 && !strncmp(l->s, "---", 3) && (l->len == 3 || l->s[3] == ' ')) {
            if (l->len > 3) {
                int b = 3, e = l->len;
                e = comment_start(l->s, b, e);
                trim(l->s, &b, &e);
                if (b != e) { fail(&p, l->lineno, "content after '---' is not supported"); free(p.L); return NULL; }
            }
            p.i = first + 1;
        }
    }
    for (int j = p.i; j < p.n; j++) {
        const yl_line *l = &p.L[j];
        if (l->indent == 0 && l->len >= 3 && (!strncmp(l->s, "---", 3) || !strncmp(l->s, "...", 3)) &&
            (l->len == 3 || l->s[3] == ' ')) {
            if (l->s[0] == '-') { fail(&p, l->lineno, "more than one document"); free(p.L); return NULL; }
            p.n = j;                   /* "...": the rest is ignored */
            break;
        }
    }
    yl_doc *d = (yl_doc *)calloc(1, sizeof(yl_doc));
    if (!d) { free(p.L); return NULL; }
    const int any = next_content(&p) >= 0;
    if (any) d->root = block_node(&p, 0);
    if (!p.failed && any && next_content(&p) >= 0)
        fail(&p, p.L[p.i].lineno, "unexpected text (indentation)");
    free(p.L);
    if (p.failed || (any && !d->root)) { yl_free(d); return NULL; }
    if (push(d, YL_EV_STREAM_START, NULL)) { yl_free(d); return NULL; }
    if (d->root) {
        if (push(d, YL_EV_DOC_START, NULL) || emit(d, d->root) || push(d, YL_EV_DOC_END, NULL)) {
            yl_free(d);
            return NULL;
        }
    }
    if (push(d, YL_EV_STREAM_END, NULL)) { yl_free(d); return NULL; }
    return d;
}

void yl_free(yl_doc *d)
{
    if (!d) return;
    node_free(d->root);
    free(d->ev);
    free(d);
}

int yl_get(const yl_doc *d, const char *path, const char *prop, const char **vals, int max)
{
    char tokbuf[1024];
    if (!d || strlen(path) >= sizeof(tokbuf)) return 0;
    strcpy(tokbuf, path);
    int pos = 0, doclevel = 0, proplevel = 0;
    int last = 0;
    char *save = NULL;
    for (char *tok = strtok_r(tokbuf, "/", &save); tok; tok = strtok_r(NULL, "/", &save)) {
        proplevel++;
        int found = 0;
        while (pos < d->nev) {
            const yl_event *e = &d->ev[pos++];
            last = e->type;
            if (e->type == YL_EV_DOC_END) break;
            if (e->type == YL_EV_STREAM_START || e->type == YL_EV_DOC_START) continue;
            if (e->type == YL_EV_MAP_START) doclevel++;
            if (e->type == YL_EV_MAP_END) doclevel--;
            if (e->type == YL_EV_SCALAR && !strcmp(e->value, tok) && doclevel == proplevel) { found = 1; break; }
            if (doclevel < proplevel) return 0;
        }
        if (!found) return 0;
    }
    (void)last;
    int mappinglevel = 0;
    while (pos < d->nev) {
        const yl_event *e = &d->ev[pos++];
        if (e->type == YL_EV_MAP_START) mappinglevel++;
        if (e->type == YL_EV_MAP_END) mappinglevel--;
        if (e->type == YL_EV_SCALAR && !strcmp(e->value, prop)) {
            if (pos >= d->nev) return 0;
            const yl_event *v = &d->ev[pos++];
            int n = 0;
            if (v->type == YL_EV_SEQ_START) {
                while (pos < d->nev && d->ev[pos].type != YL_EV_SEQ_END) {
                    if (d->ev[pos].type == YL_EV_SCALAR) {
                        if (n < max) vals[n] = d->ev[pos].value;
                        n++;
                    }
                    pos++;
                }
            } else if (v->type == YL_EV_SCALAR) {
                if (max > 0) vals[0] = v->value;
                n = 1;
            }
            return n;
        }
        if (e->type == YL_EV_MAP_END && !mappinglevel) return 0;
    }
    return 0;
}
