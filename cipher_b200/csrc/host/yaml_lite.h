/*
 * yaml_lite.h - the YAML subset of the reference's configuration files, as
 * a tree and as the event stream the reference's GetProperty walks.
 *
 * The reference reads its configuration with libyaml's event parser
 * (src/init.c:24-99).  libyaml is not part of this build; this parser
 * covers the YAML the configuration format uses: block mappings by
 * indentation, plain and quoted scalars, flow sequences ("[a, b]", nested
 * allowed), flow mappings, block sequences ("- item"), literal and folded
 * block scalars ("|", "|-", "|+", ">"), comments, document markers and
 * CRLF line ends.  Anchors, aliases, tags and multi-document streams are
 * rejected.
 */
#ifndef CIPHER_YAML_LITE_H
#define CIPHER_YAML_LITE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { YL_SCALAR = 0, YL_MAPPING = 1, YL_SEQUENCE = 2 };

typedef struct yl_node {
    int kind;
    char *value;                 /* scalar text (YL_SCALAR) */
    int n, cap;
    char **keys;                 /* mapping keys [n] (YL_MAPPING) */
    struct yl_node **kids;       /* mapping values / sequence items [n] */
} yl_node;

/* the events of libyaml's parser that GetProperty looks at */
enum { YL_EV_STREAM_START = 1, YL_EV_STREAM_END, YL_EV_DOC_START, YL_EV_DOC_END, YL_EV_SCALAR,
       YL_EV_SEQ_START, YL_EV_SEQ_END, YL_EV_MAP_START, YL_EV_MAP_END };

typedef struct yl_event {
    int type;
    const char *value;           /* YL_EV_SCALAR: points into the tree */
} yl_event;

typedef struct yl_doc {
    yl_node *root;
    yl_event *ev;
    int nev, capev;
} yl_doc;

/* parse text[len]; on error returns NULL and writes a message (line number
 * included) into err[errlen] */
yl_doc *yl_parse(const char *text, size_t len, char *err, size_t errlen);
void yl_free(yl_doc *d);

/* GetProperty (src/init.c:24-99) on the document's event stream: walks to
 * the mapping `path` ("a/b/c": each token the first scalar at its mapping
 * depth), then takes the first scalar equal to `prop` at any depth inside
 * that mapping and returns its value: the scalars of a sequence (up to the
 * first sequence end) or one scalar.  Returns the number of values (0 when
 * the mapping or the property is absent); vals[0..max) point into the tree */
int yl_get(const yl_doc *d, const char *path, const char *prop, const char **vals, int max);

#ifdef __cplusplus
}
#endif
#endif
