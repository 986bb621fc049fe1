// The part of XLA's foreign-function-interface C ABI (the structs an XLA
// custom-call handler receives and the API functions it calls) that the
// handlers in sbh_xla_ffi.cu use. The layouts are the interface XLA and a
// handler library share across the shared-library boundary (XLA's public
// xla/ffi/api/c_api.h, API version 0.1): a handler built against them works
// with any XLA runtime that speaks that version, without XLA's headers. Only
// the fields read or written here are spelled out; every struct carries its
// own struct_size, which the code checks before reading a field.
#ifndef SBH_XLA_FFI_ABI_H_
#define SBH_XLA_FFI_ABI_H_

#include <stddef.h>
#include <stdint.h>

extern "C" {

typedef struct XLA_FFI_Api XLA_FFI_Api;
typedef struct XLA_FFI_Error XLA_FFI_Error;                        // opaque, owned by XLA
typedef struct XLA_FFI_ExecutionContext XLA_FFI_ExecutionContext;  // opaque

constexpr int kXlaFfiApiMajor = 0;
constexpr int kXlaFfiApiMinor = 1;

typedef enum { XLA_FFI_Extension_Metadata = 1 } XLA_FFI_Extension_Type;

typedef struct XLA_FFI_Extension_Base {
  size_t struct_size;
  XLA_FFI_Extension_Type type;
  struct XLA_FFI_Extension_Base* next;
} XLA_FFI_Extension_Base;

typedef struct XLA_FFI_Api_Version {
  size_t struct_size;
  XLA_FFI_Extension_Base* extension_start;
  int major_version;
  int minor_version;
} XLA_FFI_Api_Version;

typedef enum {
  XLA_FFI_Error_Code_OK = 0,
  XLA_FFI_Error_Code_INVALID_ARGUMENT = 3,
  XLA_FFI_Error_Code_RESOURCE_EXHAUSTED = 8,
  XLA_FFI_Error_Code_INTERNAL = 13,
} XLA_FFI_Error_Code;

typedef enum {
  XLA_FFI_DataType_INVALID = 0,
  XLA_FFI_DataType_S32 = 4,
  XLA_FFI_DataType_U8 = 6,
  XLA_FFI_DataType_F32 = 11,
} XLA_FFI_DataType;

typedef enum { XLA_FFI_ArgType_BUFFER = 1 } XLA_FFI_ArgType;
typedef enum { XLA_FFI_RetType_BUFFER = 1 } XLA_FFI_RetType;
typedef enum {
  XLA_FFI_AttrType_ARRAY = 1,
  XLA_FFI_AttrType_DICTIONARY = 2,
  XLA_FFI_AttrType_SCALAR = 3,
  XLA_FFI_AttrType_STRING = 4,
} XLA_FFI_AttrType;

typedef enum {
  XLA_FFI_ExecutionStage_INSTANTIATE = 0,
  XLA_FFI_ExecutionStage_PREPARE = 1,
  XLA_FFI_ExecutionStage_INITIALIZE = 2,
  XLA_FFI_ExecutionStage_EXECUTE = 3,
} XLA_FFI_ExecutionStage;

typedef struct XLA_FFI_Buffer {
  size_t struct_size;
  XLA_FFI_Extension_Base* extension_start;
  XLA_FFI_DataType dtype;
  void* data;
  int64_t rank;
  int64_t* dims;
} XLA_FFI_Buffer;

typedef struct XLA_FFI_Args {
  size_t struct_size;
  XLA_FFI_Extension_Base* extension_start;
  int64_t size;
  XLA_FFI_ArgType* types;
  void** args;
} XLA_FFI_Args;

typedef struct XLA_FFI_Rets {
  size_t struct_size;
  XLA_FFI_Extension_Base* extension_start;
  int64_t size;
  XLA_FFI_RetType* types;
  void** rets;
} XLA_FFI_Rets;

typedef struct XLA_FFI_ByteSpan {
  const char* ptr;
  size_t len;
} XLA_FFI_ByteSpan;

typedef struct XLA_FFI_Scalar {
  XLA_FFI_DataType dtype;
  void* value;
} XLA_FFI_Scalar;

typedef struct XLA_FFI_Attrs {
  size_t struct_size;
  XLA_FFI_Extension_Base* extension_start;
  int64_t size;
  XLA_FFI_AttrType* types;
  XLA_FFI_ByteSpan** names;
  void** attrs;
} XLA_FFI_Attrs;

typedef struct XLA_FFI_CallFrame {
  size_t struct_size;
  XLA_FFI_Extension_Base* extension_start;
  const XLA_FFI_Api* api;
  XLA_FFI_ExecutionContext* ctx;
  XLA_FFI_ExecutionStage stage;
  XLA_FFI_Args args;
  XLA_FFI_Rets rets;
  XLA_FFI_Attrs attrs;
} XLA_FFI_CallFrame;

typedef uint32_t XLA_FFI_Handler_Traits;

typedef struct XLA_FFI_Metadata {
  size_t struct_size;
  XLA_FFI_Api_Version api_version;
  XLA_FFI_Handler_Traits traits;
} XLA_FFI_Metadata;

typedef struct XLA_FFI_Metadata_Extension {
  XLA_FFI_Extension_Base extension_base;
  XLA_FFI_Metadata* metadata;
} XLA_FFI_Metadata_Extension;

typedef struct XLA_FFI_Error_Create_Args {
  size_t struct_size;
  XLA_FFI_Extension_Base* extension_start;
  const char* message;
  XLA_FFI_Error_Code errc;
} XLA_FFI_Error_Create_Args;

typedef struct XLA_FFI_Stream_Get_Args {
  size_t struct_size;
  XLA_FFI_Extension_Base* extension_start;
  XLA_FFI_ExecutionContext* ctx;
  void* stream;  // out
} XLA_FFI_Stream_Get_Args;

typedef struct XLA_FFI_DeviceMemory_Allocate_Args {
  size_t struct_size;
  XLA_FFI_Extension_Base* extension_start;
  XLA_FFI_ExecutionContext* ctx;
  size_t size;
  size_t alignment;
  void* data;  // out
} XLA_FFI_DeviceMemory_Allocate_Args;

typedef struct XLA_FFI_DeviceMemory_Free_Args {
  size_t struct_size;
  XLA_FFI_Extension_Base* extension_start;
  XLA_FFI_ExecutionContext* ctx;
  size_t size;
  void* data;
} XLA_FFI_DeviceMemory_Free_Args;

typedef XLA_FFI_Error* XLA_FFI_Error_Create_Fn(XLA_FFI_Error_Create_Args* args);
typedef void XLA_FFI_Unused_Fn(void);
typedef XLA_FFI_Error* XLA_FFI_Stream_Get_Fn(XLA_FFI_Stream_Get_Args* args);
typedef XLA_FFI_Error* XLA_FFI_DeviceMemory_Allocate_Fn(XLA_FFI_DeviceMemory_Allocate_Args* args);
typedef XLA_FFI_Error* XLA_FFI_DeviceMemory_Free_Fn(XLA_FFI_DeviceMemory_Free_Args* args);

// The API table: the version, then one function pointer per entry point in
// XLA's order. A table shorter than a field's end (struct_size) lacks it.
struct XLA_FFI_Api {
  size_t struct_size;
  XLA_FFI_Extension_Base* extension_start;
  XLA_FFI_Api_Version api_version;
  void* internal_api;
  XLA_FFI_Error_Create_Fn* XLA_FFI_Error_Create;
  XLA_FFI_Unused_Fn* XLA_FFI_Error_GetMessage;
  XLA_FFI_Unused_Fn* XLA_FFI_Error_Destroy;
  XLA_FFI_Unused_Fn* XLA_FFI_Handler_Register;
  XLA_FFI_Stream_Get_Fn* XLA_FFI_Stream_Get;
  XLA_FFI_Unused_Fn* XLA_FFI_TypeId_Register;
  XLA_FFI_Unused_Fn* XLA_FFI_ExecutionContext_Get;
  XLA_FFI_Unused_Fn* XLA_FFI_State_Set;
  XLA_FFI_Unused_Fn* XLA_FFI_State_Get;
  XLA_FFI_DeviceMemory_Allocate_Fn* XLA_FFI_DeviceMemory_Allocate;
  XLA_FFI_DeviceMemory_Free_Fn* XLA_FFI_DeviceMemory_Free;
};

}  // extern "C"

#endif  // SBH_XLA_FFI_ABI_H_
