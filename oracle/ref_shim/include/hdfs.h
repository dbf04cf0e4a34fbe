/* hdfs.h — declarations of the libhdfs C API names the reference's HDFS
 * helpers mention, for the oracle shim (test infrastructure only).  Nothing
 * here is defined: the shim reads no HDFS path, so no call is ever made. */
#ifndef PLATO_ORACLE_SHIM_HDFS_H
#define PLATO_ORACLE_SHIM_HDFS_H
#include <fcntl.h>

#include <cstdint>
#include <ctime>
extern "C" {
typedef int32_t tSize;
typedef time_t tTime;
typedef int64_t tOffset;
typedef uint16_t tPort;
typedef enum tObjectKind { kObjectKindFile = 'F', kObjectKindDirectory = 'D' } tObjectKind;
struct hdfs_internal;
typedef struct hdfs_internal* hdfsFS;
struct hdfsFile_internal;
typedef struct hdfsFile_internal* hdfsFile;
struct hdfsBuilder;
typedef struct {
  tObjectKind mKind;
  char* mName;
  tTime mLastMod;
  tOffset mSize;
  short mReplication;
  tOffset mBlockSize;
  char* mOwner;
  char* mGroup;
  short mPermissions;
  tTime mLastAccess;
} hdfsFileInfo;
struct hdfsBuilder* hdfsNewBuilder(void);
void hdfsBuilderSetNameNode(struct hdfsBuilder*, const char*);
void hdfsBuilderSetUserName(struct hdfsBuilder*, const char*);
int hdfsBuilderConfSetStr(struct hdfsBuilder*, const char*, const char*);
hdfsFS hdfsBuilderConnect(struct hdfsBuilder*);
int hdfsDisconnect(hdfsFS);
hdfsFile hdfsOpenFile(hdfsFS, const char*, int, int, short, tSize);
int hdfsCloseFile(hdfsFS, hdfsFile);
int hdfsExists(hdfsFS, const char*);
int hdfsSeek(hdfsFS, hdfsFile, tOffset);
tOffset hdfsTell(hdfsFS, hdfsFile);
tSize hdfsRead(hdfsFS, hdfsFile, void*, tSize);
tSize hdfsWrite(hdfsFS, hdfsFile, const void*, tSize);
int hdfsFlush(hdfsFS, hdfsFile);
int hdfsFileIsOpenForWrite(hdfsFile);
int hdfsDelete(hdfsFS, const char*, int);
int hdfsMove(hdfsFS, const char*, hdfsFS, const char*);
int hdfsCreateDirectory(hdfsFS, const char*);
hdfsFileInfo* hdfsListDirectory(hdfsFS, const char*, int*);
hdfsFileInfo* hdfsGetPathInfo(hdfsFS, const char*);
void hdfsFreeFileInfo(hdfsFileInfo*, int);
}
#endif
