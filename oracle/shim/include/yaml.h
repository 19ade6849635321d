/*
 * yaml.h - the part of libyaml's event API that the reference's GetProperty
 * calls (src/init.c:24-99), as a replay of an event stream the caller
 * supplies (oracle only).
 *
 * libyaml is not installed here.  The oracle takes the events of a
 * configuration file from an independent YAML parser (PyYAML, whose event
 * model is libyaml's) and hands them to ref_config_events(); every
 * yaml_parser_set_input_string() then starts the replay from the first
 * event, which is what re-parsing the same buffer does in libyaml.
 */
#ifndef CIPHER_SHIM_YAML_H
#define CIPHER_SHIM_YAML_H
#include <stddef.h>

typedef enum yaml_event_type_e {
    YAML_NO_EVENT = 0,
    YAML_STREAM_START_EVENT,
    YAML_STREAM_END_EVENT,
    YAML_DOCUMENT_START_EVENT,
    YAML_DOCUMENT_END_EVENT,
    YAML_ALIAS_EVENT,
    YAML_SCALAR_EVENT,
    YAML_SEQUENCE_START_EVENT,
    YAML_SEQUENCE_END_EVENT,
    YAML_MAPPING_START_EVENT,
    YAML_MAPPING_END_EVENT
} yaml_event_type_t;

typedef struct yaml_event_s {
    yaml_event_type_t type;
    union {
        struct {
            unsigned char *value;
            size_t length;
        } scalar;
    } data;
} yaml_event_t;

typedef struct yaml_parser_s {
    int pos;
} yaml_parser_t;

int yaml_parser_initialize(yaml_parser_t *parser);
void yaml_parser_set_input_string(yaml_parser_t *parser, const unsigned char *input, size_t size);
int yaml_parser_parse(yaml_parser_t *parser, yaml_event_t *event);
void yaml_event_delete(yaml_event_t *event);
void yaml_parser_delete(yaml_parser_t *parser);

#endif
